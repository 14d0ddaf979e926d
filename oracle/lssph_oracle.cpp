// lssph_oracle.cpp -- CPU restatement of the LS-SPH-Benchmarks hot path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the CUDA engine and
// the timed CPU baseline of bench.py; nothing in the shipped engine links or calls it.
// It restates the reference Fortran (LS-SPH-Benchmarks, source/...) subroutine by
// subroutine, with the loop order of a single OpenMP thread, so that
//   * the cell list order is deterministic (ascending particle index within a cell,
//     then the ghost list: update_cell_mod.f90:49-93 run by one thread), and
//   * every per-particle loop (calculate_RHS, ghost, PST) is independent per particle,
//     so running it on N threads gives bit-identical results.
//
// Arithmetic conventions (the CUDA FP64 path follows the same sequence):
//   * compiled with -ffp-contract=off: no implicit FMA contraction;
//   * explicit fma() only at accumulation sites "acc = acc + a*b" (moment matrix,
//     b vectors, shift vector, dot products) and in the LU update/substitutions;
//   * Fortran integer powers x**n are evaluated as products p2=x*x, p3=p2*x, p4=p2*p2,
//     p5=p4*x, p6=p4*p2, p7=p6*x, p8=p4*p4;
//   * a division by a quantity that is invariant over a loop (h, W_ave, rho_i, zeta^2,
//     xi^2, a pivot, r in the two shift components) is a multiplication by its
//     reciprocal, as an optimising Fortran compiler under a fast floating-point model
//     (ifx's default fp-model fast=1, the reference Makefile's first option) may emit it;
//     gfortran -O2 keeps true divisions, so the reference's own bits differ between its
//     two documented builds at this level;
//   * LAPACK DGESV (LSSPH_A_mod.f90:211, shift_interpolate_mod.f90:241,
//     interpolate_LSSPH_B_mod.f90:158) is restated as Gaussian elimination with partial
//     pivoting (first max |a| pivot, reciprocal scaling of the column, right-looking
//     update, then unit-lower and upper substitutions), i.e. the reference-LAPACK
//     dgetf2/dgetrs sequence.  The reference links an unpinned MKL/LAPACK, so the
//     bits at this boundary are not pinned; tests check it against scipy's dgesv.
//
// Parity status: the kernel functions and the LS type-B interpolation are pinned by
// golden vectors generated from the reference's own Python (analysis/common/
// kernel_functions.py, analysis/common/lssph_b.py); the Fortran-only parts are pinned
// by analytic known answers (exact reproduction of quadratics, the diffusion-test
// eigenfunction, Taylor-Green decay) because no Fortran compiler exists here.

#include "../include/lssph.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr double PI = 3.14159265358979323846;  // == acos(-1.0d0)

thread_local std::string g_err;

// ---------------------------------------------------------------------------------
// Kernel functions (kernel_functions_mod.f90:26-146)
// ---------------------------------------------------------------------------------
double kernel_norm(int kt, double h) {
    const double hh = h * h;
    switch (kt) {
        case 1: return 5.0 / ((14.0 * PI) * hh);
        case 2: return 7.0 / ((478.0 * PI) * hh);
        case 3: return 7.0 / ((4.0 * PI) * hh);
        case 4: return 9.0 / ((4.0 * PI) * hh);
        default: return 39.0 / ((14.0 * PI) * hh);
    }
}

// kernel_functions_mod.f90:26-81
double cal_W(int kt, double r, double h) {
    const double q = r * (1.0 / h);
    double W = 0.0;
    if (kt == 1) {
        const double a = 2.0 - q, b = 1.0 - q;
        const double a3 = (a * a) * a, b3 = (b * b) * b;
        if (0.0 <= q && q <= 1.0) W = a3 - 4.0 * b3;
        else if (1.0 < q && q <= 2.0) W = a3;
    } else if (kt == 2) {
        const double a = 3.0 - q, b = 2.0 - q, c = 1.0 - q;
        const double a2 = a * a, b2 = b * b, c2 = c * c;
        const double a5 = (a2 * a2) * a, b5 = (b2 * b2) * b, c5 = (c2 * c2) * c;
        if (0.0 <= q && q <= 1.0) W = (a5 - 6.0 * b5) + 15.0 * c5;
        else if (1.0 < q && q <= 2.0) W = a5 - 6.0 * b5;
        else if (2.0 < q && q <= 3.0) W = a5;
    } else if (kt == 3) {
        if (0.0 <= q && q <= 2.0) {
            const double t = 1.0 - 0.5 * q, t2 = t * t, t4 = t2 * t2;
            W = t4 * (1.0 + 2.0 * q);
        }
    } else if (kt == 4) {
        if (0.0 <= q && q <= 2.0) {
            const double t = 1.0 - 0.5 * q, t2 = t * t, t4 = t2 * t2, t6 = t4 * t2;
            W = t6 * ((1.0 + 3.0 * q) + (35.0 * (q * q)) / 12.0);
        }
    } else {
        if (0.0 <= q && q <= 2.0) {
            const double t = 1.0 - 0.5 * q, t2 = t * t, t4 = t2 * t2, t8 = t4 * t4;
            const double q2 = q * q, q3 = q2 * q;
            W = t8 * (((1.0 + 4.0 * q) + (25.0 * q2) / 4.0) + 4.0 * q3);
        }
    }
    return kernel_norm(kt, h) * W;
}

// kernel_functions_mod.f90:87-146
double cal_dW(int kt, double r, double h) {
    const double ih = 1.0 / h;
    const double q = r * ih;
    double dW = 0.0;
    const double nrm = kernel_norm(kt, h);
    if (kt == 1) {
        const double a = 2.0 - q, b = 1.0 - q;
        if (0.0 <= q && q <= 1.0) dW = a * a - 4.0 * (b * b);
        else if (1.0 < q && q <= 2.0) dW = a * a;
        return (nrm * dW) * (-3.0 / h);
    } else if (kt == 2) {
        const double a = 3.0 - q, b = 2.0 - q, c = 1.0 - q;
        const double a2 = a * a, b2 = b * b, c2 = c * c;
        const double a4 = a2 * a2, b4 = b2 * b2, c4 = c2 * c2;
        if (0.0 <= q && q <= 1.0) dW = (a4 - 6.0 * b4) + 15.0 * c4;
        else if (1.0 < q && q <= 2.0) dW = a4 - 6.0 * b4;
        else if (2.0 < q && q <= 3.0) dW = a4;
        return (nrm * dW) * (-5.0 / h);
    } else if (kt == 3) {
        if (0.0 <= q && q <= 2.0) {
            const double t = 1.0 - 0.5 * q, t2 = t * t, t3 = t2 * t, t4 = t2 * t2;
            dW = -(2.0 * t3) * (1.0 + 2.0 * q) + 2.0 * t4;
        }
    } else if (kt == 4) {
        if (0.0 <= q && q <= 2.0) {
            const double t = 1.0 - 0.5 * q, t2 = t * t, t4 = t2 * t2, t5 = t4 * t, t6 = t4 * t2;
            dW = -(3.0 * t5) * ((1.0 + 3.0 * q) + (35.0 * (q * q)) / 12.0)
                 + t6 * (3.0 + (35.0 * q) / 6.0);
        }
    } else {
        if (0.0 <= q && q <= 2.0) {
            const double t = 1.0 - 0.5 * q, t2 = t * t, t4 = t2 * t2, t6 = t4 * t2,
                         t7 = t6 * t, t8 = t4 * t4;
            const double q2 = q * q, q3 = q2 * q;
            dW = -(4.0 * t7) * (((1.0 + 4.0 * q) + (25.0 * q2) / 4.0) + 4.0 * q3)
                 + t8 * ((4.0 + (25.0 * q) / 2.0) + 12.0 * q2);
        }
    }
    return (nrm * dW) * ih;
}

// ---------------------------------------------------------------------------------
// DGESV restatement: Gaussian elimination with partial pivoting on an n x n matrix
// stored column-major (A[i + j*n]) and n x nrhs right-hand sides (B[i + k*n]).
// Returns INFO as LAPACK does (0, or the 1-based index of the first zero pivot).
// ---------------------------------------------------------------------------------
int gepp_solve(int n, int nrhs, double* A, double* B) {
    int info = 0;
    double rpiv[32];   // reciprocal pivots, reused by the back substitution
    for (int k = 0; k < n; ++k) {
        int p = k;
        double amax = std::fabs(A[k + k * n]);
        for (int i = k + 1; i < n; ++i) {
            const double a = std::fabs(A[i + k * n]);
            if (a > amax) { amax = a; p = i; }
        }
        if (A[p + k * n] != 0.0) {
            if (p != k) {
                for (int j = 0; j < n; ++j) std::swap(A[k + j * n], A[p + j * n]);
                for (int c = 0; c < nrhs; ++c) std::swap(B[k + c * n], B[p + c * n]);
            }
            const double rp = 1.0 / A[k + k * n];
            for (int i = k + 1; i < n; ++i) A[i + k * n] = A[i + k * n] * rp;
        } else if (info == 0) {
            info = k + 1;
        }
        rpiv[k] = 1.0 / A[k + k * n];
        for (int j = k + 1; j < n; ++j)
            for (int i = k + 1; i < n; ++i)
                A[i + j * n] = std::fma(-A[i + k * n], A[k + j * n], A[i + j * n]);
    }
    for (int c = 0; c < nrhs; ++c) {
        double* b = B + c * n;
        for (int k = 0; k < n; ++k)
            for (int i = k + 1; i < n; ++i) b[i] = std::fma(-b[k], A[i + k * n], b[i]);
        for (int k = n - 1; k >= 0; --k) {
            b[k] = b[k] * rpiv[k];
            for (int i = 0; i < k; ++i) b[i] = std::fma(-b[k], A[i + k * n], b[i]);
        }
    }
    return info;
}

// Taylor basis of LS-SPH type A (LSSPH_A_mod.f90:140-172); k = max order, returns q.
int basis_A(int k, double x, double y, const double* ih, double* a) {
    a[0] = x * ih[0];
    a[1] = y * ih[0];
    if (k < 2) return 2;
    const double x2 = x * x, y2 = y * y;
    a[2] = (0.5 * x2) * ih[1];
    a[3] = (0.5 * y2) * ih[1];
    a[4] = (x * y) * ih[1];
    if (k < 3) return 5;
    const double x3 = x2 * x, y3 = y2 * y;
    a[5] = ((1.0 / 6.0) * x3) * ih[2];
    a[6] = ((1.0 / 6.0) * y3) * ih[2];
    a[7] = ((0.5 * x2) * y) * ih[2];
    a[8] = ((0.5 * y2) * x) * ih[2];
    if (k < 4) return 9;
    const double x4 = x2 * x2, y4 = y2 * y2;
    a[9] = ((1.0 / 24.0) * x4) * ih[3];
    a[10] = ((1.0 / 24.0) * y4) * ih[3];
    a[11] = (((1.0 / 6.0) * x3) * y) * ih[3];
    a[12] = (((1.0 / 6.0) * y3) * x) * ih[3];
    a[13] = (((1.0 / 4.0) * x2) * y2) * ih[3];
    if (k < 5) return 14;
    const double x5 = x4 * x, y5 = y4 * y;
    a[14] = ((1.0 / 120.0) * x5) * ih[4];
    a[15] = ((1.0 / 120.0) * y5) * ih[4];
    a[16] = (((1.0 / 24.0) * x4) * y) * ih[4];
    a[17] = (((1.0 / 24.0) * y4) * x) * ih[4];
    a[18] = (((1.0 / 12.0) * x3) * y2) * ih[4];
    a[19] = (((1.0 / 12.0) * y3) * x2) * ih[4];
    return 20;
}

int order_of_model(int sph_model) {  // LSSPH_A_mod.f90:46-56
    switch (sph_model) {
        case 4: return 3;
        case 5: return 4;
        case 6: return 5;
        default: return 2;
    }
}

// ---------------------------------------------------------------------------------
// SplitMix64 jitter source (the reference draws from a clock-seeded Fortran RNG,
// impose_initial_conditions_mod.f90:43-60; a seeded counter RNG stands in for it).
// ---------------------------------------------------------------------------------
struct SplitMix64 {
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

// =====================================================================================
// State: SP_type, VM_type and Cell_type of global_types.f90:78-124 (0-based particles,
// 1-based cell ids as in the Fortran).
// =====================================================================================
struct orc_state {
    lssph_params p;
    int num_total = 0, num_int = 0, num_ext = 0;
    bool has_tem = false;
    std::vector<int> ptype;
    std::vector<double> x, y, u, v, rho, pre, tem;
    std::vector<double> x_old, y_old, u_old, v_old, rho_old, tem_old;
    std::vector<double> x_new, y_new, u_new, v_new, rho_new, tem_new;
    std::vector<double> RHS_u, RHS_v, RHS_rho, RHS_tem, f_previous;
    std::vector<int> vm_ptype, vm_pair;
    std::vector<double> vm_x, vm_y, vm_u, vm_v, vm_pre, vm_tem, vm_nx, vm_ny;
    int idx_x_max = 0, idx_y_max = 0, idx_max = 0, capacity = 0, list_cap = 0;
    std::vector<int> idx_SP, num_SP, num_WL, neighbors, list, list_WL, idx_VM;
    // periodic domain: cell width, and the position shift (+-L or 0) of each neighbour cell
    double inv_cw = 0.0;
    std::vector<double> nshift_x, nshift_y;
    int error = 0;
};

namespace {

void set_err(orc_state* s, int code, const std::string& m) {
    if (s && s->error == 0) s->error = code;
    g_err = m;
}

// init_param_mod.f90:92-199
void init_param(lssph_params* p) {
    p->total_step = (std::string(p->read_name) == "new") ? p->end_step : p->end_step - p->start_step;
    p->dx = p->len_x / (double)p->num_x;
    p->SP_mass = p->rho_ref * (p->dx * p->dx);
    p->h = p->coe_h * p->dx;
    p->h_eff = (p->kernel_type == 2) ? 3.0 * p->h : 2.0 * p->h;
    p->W_ave = cal_W(p->kernel_type, p->dx, p->h);
    p->num_WL = (int)std::ceil(p->h_eff / p->dx);
    if (p->periodic) p->num_WL = 0;   // periodic extension: no wall layers
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

// setup_closed_box_mod.f90:23-237 + impose_initial_conditions_mod.f90
void setup_closed_box(orc_state* s) {
    const lssph_params& p = s->p;
    const int nxf = p.num_x + 2 * p.num_WL, nyf = p.num_y + 2 * p.num_WL, nf = nxf * nyf;
    std::vector<double> xs(nf), ys(nf);
    xs[0] = p.dx / 2.0;
    ys[0] = p.dx / 2.0;
    for (int i = 1; i < nf; ++i) {
        if (i < nxf) { xs[i] = xs[i - 1] + p.dx; ys[i] = ys[i - 1]; }
        else { xs[i] = xs[i - nxf]; ys[i] = ys[i - nxf] + p.dx; }
    }
    const double x_min = 0.0 + p.WL_thick, x_max = p.len_x + p.WL_thick;
    const double y_min = 0.0 + p.WL_thick, y_max = p.len_y + p.WL_thick;
    std::vector<double> xi, yi, xe, ye;
    for (int i = 0; i < nf; ++i) {
        if (x_min < xs[i] && x_max > xs[i] && y_min < ys[i] && y_max > ys[i]) { xi.push_back(xs[i]); yi.push_back(ys[i]); }
        else { xe.push_back(xs[i]); ye.push_back(ys[i]); }
    }
    s->num_int = (int)xi.size();
    s->num_ext = (int)xe.size();
    s->num_total = s->num_int + s->num_ext;
    const int N = s->num_total;
    s->ptype.assign(N, 0);
    s->x.assign(N, 0.0); s->y.assign(N, 0.0); s->u.assign(N, 0.0); s->v.assign(N, 0.0);
    s->rho.assign(N, 0.0); s->pre.assign(N, 0.0); s->tem.assign(N, 0.0);
    for (int i = 0; i < s->num_int; ++i) { s->x[i] = xi[i]; s->y[i] = yi[i]; }
    for (int i = 0; i < s->num_ext; ++i) { s->x[s->num_int + i] = xe[i]; s->y[s->num_int + i] = ye[i]; }
    for (int i = s->num_int; i < N; ++i) {
        s->rho[i] = p.rho_ref;
        int t;
        if (s->y[i] < y_min) { t = 1; if (s->x[i] < x_min) t = 5; if (s->x[i] > x_max) t = 6; }
        else if (s->y[i] > y_max) { t = 2; if (s->x[i] < x_min) t = 7; if (s->x[i] > x_max) t = 8; }
        else if (s->x[i] < x_min) t = 3;
        else if (s->x[i] > x_max) t = 4;
        else { t = 10; set_err(s, LSSPH_E_BAD_PARAM, "setup_closed_box: unclassified ghost"); }
        s->ptype[i] = t;
    }
}

void impose_ic(orc_state* s) {
    const lssph_params& p = s->p;
    const int n = s->num_int;
    if (p.target_problem == 1) {  // impose_initial_conditions_mod.f90:24-62
        std::fill(s->rho.begin(), s->rho.end(), p.rho_ref);
        std::fill(s->u.begin(), s->u.end(), 0.0);
        std::fill(s->pre.begin(), s->pre.end(), 0.0);
        std::fill(s->v.begin(), s->v.end(), 0.0);
        SplitMix64 rng{p.seed};
        for (int i = 0; i < n; ++i) {
            double r = rng.uniform();
            s->x[i] = s->x[i] + (p.pos_pert * p.dx) * (2.0 * r - 1.0);
            r = rng.uniform();
            s->y[i] = s->y[i] + (p.pos_pert * p.dx) * (2.0 * r - 1.0);
        }
        if (p.periodic) {   // periodic extension: free decay of sin(2 pi x) sin(2 pi y)
            for (int i = 0; i < n; ++i)
                s->u[i] = std::sin(((2.0 * PI) * s->x[i]) / p.len_x) * std::sin(((2.0 * PI) * s->y[i]) / p.len_y);
        }
    } else if (p.target_problem == 2) {  // :68-96
        const double a = (double)p.tg_a, b = (double)p.tg_b, Lx = p.len_x, Ly = p.len_y;
        const double ratio = (a * Ly) / (b * Lx);
        for (int i = 0; i < n; ++i) {
            const double xx = s->x[i] - p.WL_thick, yy = s->y[i] - p.WL_thick;
            s->u[i] = (1.0 * std::sin(((a * PI) * xx) / Lx)) * std::cos(((b * PI) * yy) / Ly);
            s->v[i] = ((-1.0 * ratio) * std::cos(((a * PI) * xx) / Lx)) * std::sin(((b * PI) * yy) / Ly);
            s->pre[i] = ((0.25 * p.rho_ref) * 1.0) *
                        (std::cos((((2.0 * a) * PI) * xx) / Lx) + (ratio * ratio) * std::cos((((2.0 * b) * PI) * yy) / Ly));
            s->rho[i] = p.rho_ref + s->pre[i] / (p.sound_speed * p.sound_speed);
        }
    } else if (p.target_problem == 3) {  // :102-111
        std::fill(s->rho.begin(), s->rho.end(), p.rho_ref);
        std::fill(s->pre.begin(), s->pre.end(), 0.0);
        std::fill(s->u.begin(), s->u.end(), 0.0);
        std::fill(s->v.begin(), s->v.end(), 0.0);
    } else {  // :117-145
        std::fill(s->rho.begin(), s->rho.end(), p.rho_ref);
        std::fill(s->pre.begin(), s->pre.end(), 0.0);
        std::fill(s->u.begin(), s->u.end(), 0.0);
        std::fill(s->v.begin(), s->v.end(), 0.0);
        for (int i = 0; i < n; ++i) {
            const double xx = s->x[i] - p.WL_thick, yy = s->y[i] - p.WL_thick;
            s->tem[i] = -(p.delta_tem / p.len_y) * yy + p.tem_bottom;
            if (yy <= 0.1 * p.len_y) s->tem[i] = s->tem[i] + (1.0e-2 * p.delta_tem) * std::cos((PI * xx) / p.len_x);
        }
    }
}

void alloc_work(orc_state* s) {
    const int n = s->num_int;
    for (auto* vec : {&s->x_old, &s->y_old, &s->u_old, &s->v_old, &s->rho_old, &s->tem_old,
                      &s->x_new, &s->y_new, &s->u_new, &s->v_new, &s->rho_new, &s->tem_new,
                      &s->RHS_u, &s->RHS_v, &s->RHS_rho, &s->RHS_tem})
        vec->assign(n, 0.0);
    s->f_previous.assign(n, 1.0);  // setup_closed_box_mod.f90:160-163
    if ((int)s->tem.size() != s->num_total) s->tem.assign(s->num_total, 0.0);
}

// init_virtual_markers_mod.f90:23-141
void init_virtual_markers(orc_state* s) {
    const lssph_params& p = s->p;
    const int ne = s->num_ext;
    s->vm_ptype.assign(ne, 0); s->vm_pair.assign(ne, 0);
    for (auto* vec : {&s->vm_x, &s->vm_y, &s->vm_u, &s->vm_v, &s->vm_pre, &s->vm_tem, &s->vm_nx, &s->vm_ny})
        vec->assign(ne, 0.0);
    const double x_min = 0.0 + p.WL_thick, x_max = p.len_x + p.WL_thick;
    const double y_min = 0.0 + p.WL_thick, y_max = p.len_y + p.WL_thick;
    const double r2 = 1.0 / std::sqrt(2.0);
    for (int me = 0; me < ne; ++me) {
        const int you = s->num_int + me;
        s->vm_pair[me] = you;
        const int t = s->ptype[you];
        s->vm_ptype[me] = t;
        double vx = s->x[you], vy = s->y[you], nx = 0.0, ny = 0.0;
        switch (t) {
            case 1: vy = 2.0 * y_min - s->y[you]; ny = -1.0; break;
            case 2: vy = 2.0 * y_max - s->y[you]; ny = 1.0; break;
            case 3: vx = 2.0 * x_min - s->x[you]; nx = -1.0; break;
            case 4: vx = 2.0 * x_max - s->x[you]; nx = 1.0; break;
            case 5: vx = 2.0 * x_min - s->x[you]; vy = 2.0 * y_min - s->y[you]; nx = -r2; ny = -r2; break;
            case 6: vx = 2.0 * x_max - s->x[you]; vy = 2.0 * y_min - s->y[you]; nx = r2; ny = -r2; break;
            case 7: vx = 2.0 * x_min - s->x[you]; vy = 2.0 * y_max - s->y[you]; nx = -r2; ny = r2; break;
            case 8: vx = 2.0 * x_max - s->x[you]; vy = 2.0 * y_max - s->y[you]; nx = r2; ny = r2; break;
            default: set_err(s, LSSPH_E_BAD_PARAM, "init_virtual_markers: bad ghost ptype");
        }
        s->vm_x[me] = vx; s->vm_y[me] = vy; s->vm_nx[me] = nx; s->vm_ny[me] = ny;
    }
}

// Cell of a position in a periodic square: an even number of cells of width L / n >= h_eff,
// x in (0, L] -> ceil(x / width), clamped against rounding at x = L.
int periodic_cell(const orc_state* s, double x) {
    int c = (int)std::ceil(x * s->inv_cw);
    return c < 1 ? 1 : (c > s->idx_x_max ? s->idx_x_max : c);
}

// Periodic position wrap into (0, L].
inline double wrap_pos(double x, double L) { return x <= 0.0 ? x + L : (x > L ? x - L : x); }

// init_cell_mod.f90:23-184 (+ the periodic extension)
void init_cell(orc_state* s) {
    const lssph_params& p = s->p;
    const double xm = p.len_x + 2.0 * p.WL_thick, ym = p.len_y + 2.0 * p.WL_thick;
    s->idx_x_max = (int)std::ceil(xm / p.h_eff);
    s->idx_y_max = (int)std::ceil(ym / p.h_eff);
    if (p.periodic) {
        const int n = 2 * (int)std::floor(p.len_x / (2.0 * p.h_eff));
        s->idx_x_max = n;
        s->idx_y_max = n;
        s->inv_cw = 1.0 / (p.len_x / (double)n);
    }
    s->idx_max = s->idx_x_max * s->idx_y_max;
    const int nc = s->idx_max;
    s->idx_SP.assign(s->num_total, 0);
    s->num_SP.assign(nc + 1, 0);
    s->num_WL.assign(nc + 1, 0);
    s->idx_VM.assign(s->num_ext, 0);
    s->neighbors.assign(9 * (nc + 1), 0);
    for (int me = 0; me < s->num_total; ++me) {
        int cx = (int)std::ceil(s->x[me] / p.h_eff), cy = (int)std::ceil(s->y[me] / p.h_eff);
        if (p.periodic) { cx = periodic_cell(s, s->x[me]); cy = periodic_cell(s, s->y[me]); }
        int c = cx + (cy - 1) * s->idx_x_max;
        if (cx < 1 || cx > s->idx_x_max || cy < 1 || cy > s->idx_y_max) {
            set_err(s, LSSPH_E_OUT_OF_DOMAIN, "init_cell: particle outside the cell grid");
            c = 1;
        }
        s->idx_SP[me] = c;
        s->num_SP[c] += 1;
    }
    s->capacity = *std::max_element(s->num_SP.begin() + 1, s->num_SP.end());
    s->list_cap = 2 * s->capacity;
    s->list.assign((size_t)s->list_cap * (nc + 1), 0);
    s->list_WL.assign((size_t)s->list_cap * (nc + 1), 0);
    for (int me = s->num_int; me < s->num_total; ++me) {
        const int c = s->idx_SP[me];
        s->num_WL[c] += 1;
        s->list_WL[(size_t)c * s->list_cap + (s->num_WL[c] - 1)] = me;
    }
    s->nshift_x.assign(9 * (nc + 1), 0.0);
    s->nshift_y.assign(9 * (nc + 1), 0.0);
    for (int c = 1; c <= nc; ++c) {
        const int cx = (c - 1) % s->idx_x_max + 1, cy = (c - 1) / s->idx_x_max + 1;
        int k = 0;
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx) {
                int yx = cx + dx, yy = cy + dy;
                if (p.periodic) {   // wrap; the neighbour's positions appear shifted by -+L
                    if (yx < 1) { yx += s->idx_x_max; s->nshift_x[9 * c + k] = -p.len_x; }
                    if (yx > s->idx_x_max) { yx -= s->idx_x_max; s->nshift_x[9 * c + k] = p.len_x; }
                    if (yy < 1) { yy += s->idx_y_max; s->nshift_y[9 * c + k] = -p.len_y; }
                    if (yy > s->idx_y_max) { yy -= s->idx_y_max; s->nshift_y[9 * c + k] = p.len_y; }
                }
                s->neighbors[9 * c + k] = (yx < 1 || yx > s->idx_x_max || yy < 1 || yy > s->idx_y_max)
                                              ? 0 : yx + (yy - 1) * s->idx_x_max;
                ++k;
            }
    }
    for (int me = 0; me < s->num_ext; ++me) {
        const int cx = (int)std::ceil(s->vm_x[me] / p.h_eff), cy = (int)std::ceil(s->vm_y[me] / p.h_eff);
        s->idx_VM[me] = cx + (cy - 1) * s->idx_x_max;
    }
}

// update_cell_mod.f90:21-97, in the order one OpenMP thread produces
void update_cell(orc_state* s) {
    const double inv_h_eff = 1.0 / s->p.h_eff;
    const int nc = s->idx_max;
    for (int c = 1; c <= nc; ++c) s->num_SP[c] = 0;
    for (int me = 0; me < s->num_int; ++me) {
        int cx = (int)std::ceil(s->x[me] * inv_h_eff), cy = (int)std::ceil(s->y[me] * inv_h_eff);
        if (s->p.periodic) { cx = periodic_cell(s, s->x[me]); cy = periodic_cell(s, s->y[me]); }
        int c = cx + (cy - 1) * s->idx_x_max;
        if (cx < 1 || cx > s->idx_x_max || cy < 1 || cy > s->idx_y_max) {
            set_err(s, LSSPH_E_OUT_OF_DOMAIN, "update_cell: particle outside the cell grid");
            continue;
        }
        s->idx_SP[me] = c;
        const int cnt = ++s->num_SP[c];
        if (cnt > s->list_cap) { set_err(s, LSSPH_E_CELL_OVERFLOW, "update_cell: cell list overflow"); s->num_SP[c]--; continue; }
        s->list[(size_t)c * s->list_cap + (cnt - 1)] = me;
    }
    for (int c = 1; c <= nc; ++c) {
        const int nw = s->num_WL[c];
        if (nw > 0) {
            const int st = s->num_SP[c];
            if (st + nw > s->list_cap) { set_err(s, LSSPH_E_CELL_OVERFLOW, "update_cell: cell list overflow"); continue; }
            for (int k = 0; k < nw; ++k)
                s->list[(size_t)c * s->list_cap + st + k] = s->list_WL[(size_t)c * s->list_cap + k];
            s->num_SP[c] = st + nw;
        }
    }
}

// Iterate the candidate list of cell `my_cell` in reference order (9 cells, list order):
// f(you, sx, sy) with the position shift of you's cell (0 in the closed box; -+L across a
// periodic boundary), so that x_j + sx - x_i is the pair offset.
template <class F>
inline void for_candidates(const orc_state* s, int my_cell, F&& f) {
    for (int k = 0; k < 9; ++k) {
        const int c = s->neighbors[9 * my_cell + k];
        if (c == 0) continue;
        const int n = s->num_SP[c];
        const int* L = &s->list[(size_t)c * s->list_cap];
        const double sx = s->nshift_x[9 * my_cell + k], sy = s->nshift_y[9 * my_cell + k];
        for (int t = 0; t < n; ++t) f(L[t], sx, sy);
    }
}

// Problem 1 source 2 pi^2 sin(pi (x - WL)) cos(pi (y - WL)) (LSSPH_A_mod.f90:247); the
// periodic extension is source-free (0.0, added all the same).
inline double p1_source(const lssph_params& p, double x, double y) {
    if (p.periodic) return 0.0;
    return ((2.0 * (PI * PI)) * std::sin(PI * (x - p.WL_thick))) * std::cos(PI * (y - p.WL_thick));
}

// LSSPH_A_mod.f90:26-271
void LSSPH_A(orc_state* s, int me) {
    const lssph_params& p = s->p;
    const int k = order_of_model(p.sph_model);
    int q = 5;
    double ih[5];
    const double h = p.h, h_eff_sq = p.h_eff * p.h_eff, SP_mass = p.SP_mass;
    ih[0] = 1.0 / h;
    for (int i = 1; i < k; ++i) ih[i] = ih[i - 1] / h;
    const int nb = s->has_tem ? 5 : 4;
    double M[400] = {0}, b[100] = {0}, a[20] = {0};
    const double my_x = s->x[me], my_y = s->y[me], my_u = s->u[me], my_v = s->v[me];
    const double my_rho = s->rho[me], my_pre = s->pre[me], my_tem = s->has_tem ? s->tem[me] : 0.0;
    int num_neighbors = 0;
    const int qq = (k == 2) ? 5 : (k == 3) ? 9 : (k == 4) ? 14 : 20;
    q = qq;
    for_candidates(s, s->idx_SP[me], [&](int you, double sx, double sy) {
        if (me == you) return;
        const double x_ji = (s->x[you] + sx) - my_x, y_ji = (s->y[you] + sy) - my_y;
        const double r2 = x_ji * x_ji + y_ji * y_ji;
        if (r2 > h_eff_sq) return;
        const double r = std::sqrt(r2);
        const double W = cal_W(p.kernel_type, r, h);
        ++num_neighbors;
        const double V_j = SP_mass / s->rho[you];
        const double VW = V_j * W;
        basis_A(k, x_ji, y_ji, ih, a);
        double df[5];
        df[0] = s->u[you] - my_u; df[1] = s->v[you] - my_v; df[2] = s->rho[you] - my_rho;
        df[3] = s->pre[you] - my_pre;
        if (nb == 5) df[4] = s->tem[you] - my_tem;
        for (int i = 0; i < q; ++i) {
            const double VW_a = VW * a[i];
            for (int c = 0; c < nb; ++c) b[i + c * q] = std::fma(VW_a, df[c], b[i + c * q]);
            for (int j = 0; j <= i; ++j) M[j + i * q] = std::fma(VW_a, a[j], M[j + i * q]);
        }
    });
    for (int i = 0; i < q - 1; ++i)
        for (int j = i + 1; j < q; ++j) M[j + i * q] = M[i + j * q];
    double d[5][5] = {{0}};
    if (num_neighbors >= q) {
        if (gepp_solve(q, nb, M, b) != 0) set_err(s, LSSPH_E_SINGULAR, "LSSPH_A: singular moment matrix");
        for (int c = 0; c < nb; ++c) {
            d[c][0] = b[0 + c * q] * ih[0];
            d[c][1] = b[1 + c * q] * ih[0];
            d[c][2] = b[2 + c * q] * ih[1];
            d[c][3] = b[3 + c * q] * ih[1];
            d[c][4] = b[4 + c * q] * ih[1];
        }
    }
    const double* du = d[0];
    const double* dv = d[1];
    const double* drho = d[2];
    const double* dpre = d[3];
    const double* dtem = d[4];
    if (p.target_problem == 1) {
        s->RHS_u[me] = (du[2] + du[3]) + p1_source(p, my_x, my_y);
    } else {
        const double delta = ((p.coe_delta_sph * p.sound_speed) * h) * p.zeta_RSST;
        const double irho = 1.0 / my_rho;
        double Rr = -(my_rho * (du[0] + dv[1])) + delta * (drho[2] + drho[3]);
        double Ru = -(dpre[0] * irho) + (p.vis_ref * irho) * (du[2] + du[3]);
        double Rv = -(dpre[1] * irho) + (p.vis_ref * irho) * (dv[2] + dv[3]);
        Rr = Rr * (1.0 / (p.zeta_RSST * p.zeta_RSST));
        if (p.target_problem == 4) {
            const double ixi2 = 1.0 / (p.xi_VIM * p.xi_VIM);
            Rv = Rv + ((p.alpha_ref * (my_tem - p.tem_ave)) * p.gravity);
            Ru = Ru * ixi2;
            Rv = Rv * ixi2;
            s->RHS_tem[me] = p.thermal_dif * (dtem[2] + dtem[3]);
        }
        s->RHS_rho[me] = Rr; s->RHS_u[me] = Ru; s->RHS_v[me] = Rv;
    }
}

// classical_SPH_mod.f90:26-169 (SPH_MODEL 1: sum model, 2: difference model)
void classical_SPH(orc_state* s, int me) {
    const lssph_params& p = s->p;
    const double h = p.h, h_eff_sq = p.h_eff * p.h_eff, SP_mass = p.SP_mass;
    const double my_x = s->x[me], my_y = s->y[me], my_u = s->u[me], my_v = s->v[me];
    const double my_rho = s->rho[me], my_pre = s->pre[me], my_tem = s->has_tem ? s->tem[me] : 0.0;
    double du_dx = 0, dv_dy = 0, dp_dx = 0, dp_dy = 0, Lu = 0, Lv = 0, Lt = 0, Lr = 0;
    for_candidates(s, s->idx_SP[me], [&](int you, double sx, double sy) {
        if (me == you) return;
        const double x_ij = my_x - (s->x[you] + sx), y_ij = my_y - (s->y[you] + sy);
        const double r2 = x_ij * x_ij + y_ij * y_ij;
        if (r2 > h_eff_sq) return;
        const double r = std::sqrt(r2);
        const double dW = cal_dW(p.kernel_type, r, h);
        const double V_j = SP_mass / s->rho[you];
        const double gx = ((dW * x_ij) / r) * V_j, gy = ((dW * y_ij) / r) * V_j;
        du_dx = std::fma(gx, s->u[you] - my_u, du_dx);
        dv_dy = std::fma(gy, s->v[you] - my_v, dv_dy);
        if (p.sph_model == 1) {
            dp_dx = std::fma(gx, s->pre[you] + my_pre, dp_dx);
            dp_dy = std::fma(gy, s->pre[you] + my_pre, dp_dy);
        } else {
            dp_dx = std::fma(gx, s->pre[you] - my_pre, dp_dx);
            dp_dy = std::fma(gy, s->pre[you] - my_pre, dp_dy);
        }
        const double L = ((2.0 * V_j) * dW) / r;
        Lu = std::fma(L, my_u - s->u[you], Lu);
        Lv = std::fma(L, my_v - s->v[you], Lv);
        if (s->has_tem) Lt = std::fma(L, my_tem - s->tem[you], Lt);
        Lr = std::fma(L, my_rho - s->rho[you], Lr);
    });
    if (p.target_problem == 1) {
        s->RHS_u[me] = Lu + p1_source(p, my_x, my_y);
    } else {
        const double delta = ((p.coe_delta_sph * p.sound_speed) * h) * p.zeta_RSST;
        double Rr = -(my_rho * (du_dx + dv_dy)) + delta * Lr;
        double Ru = -(dp_dx / my_rho) + (p.vis_ref / my_rho) * Lu;
        double Rv = -(dp_dy / my_rho) + (p.vis_ref / my_rho) * Lv;
        Rr = Rr / (p.zeta_RSST * p.zeta_RSST);
        if (p.target_problem == 4) {
            Rv = Rv + ((p.alpha_ref * (my_tem - p.tem_ave)) * p.gravity);
            Ru = Ru / (p.xi_VIM * p.xi_VIM);
            Rv = Rv / (p.xi_VIM * p.xi_VIM);
            s->RHS_tem[me] = p.thermal_dif * Lt;
        }
        s->RHS_rho[me] = Rr; s->RHS_u[me] = Ru; s->RHS_v[me] = Rv;
    }
}

// calculate_RHS_mod.f90:29-52
void calculate_RHS(orc_state* s) {
    const int n = s->num_int;
    const bool classical = s->p.sph_model <= 2;
#pragma omp parallel for schedule(static)
    for (int me = 0; me < n; ++me) {
        if (classical) classical_SPH(s, me);
        else LSSPH_A(s, me);
    }
}

// LS type-B interpolation at (my_x, my_y) over the fluid candidates produced by
// `cands` (interpolate_LSSPH_B_mod.f90:136-255).  q = 3 (WALL_MODEL 2) or 6 (3);
// nb values per candidate from `vals(you, c)`.  Returns num_neighbors; out[c] = b(1,c).
template <class Cands, class Vals>
int lssph_b_point(const lssph_params& p, int q, int nb, double my_x, double my_y, Cands&& cands,
                  const double* X, const double* Y, const double* RHO, Vals&& vals, double* out, int* info) {
    const double h = p.h, h_eff_sq = p.h_eff * p.h_eff, SP_mass = p.SP_mass;
    const double inv_h = 1.0 / h, inv_h2 = inv_h * inv_h;
    double M[36] = {0}, b[24] = {0}, a[6] = {1.0, 0, 0, 0, 0, 0};
    int num_neighbors = 0;
    cands([&](int you) {
        const double x_ji = X[you] - my_x, y_ji = Y[you] - my_y;
        const double r2 = x_ji * x_ji + y_ji * y_ji;
        if (r2 > h_eff_sq) return;
        const double r = std::sqrt(r2);
        const double W = cal_W(p.kernel_type, r, h);
        ++num_neighbors;
        const double V_j = SP_mass / RHO[you];
        const double VW = V_j * W;
        a[1] = x_ji * inv_h;
        a[2] = y_ji * inv_h;
        if (q == 6) {
            a[3] = ((x_ji * x_ji) * 0.5) * inv_h2;
            a[4] = (x_ji * y_ji) * inv_h2;
            a[5] = ((y_ji * y_ji) * 0.5) * inv_h2;
        }
        double f[4];
        for (int c = 0; c < nb; ++c) f[c] = vals(you, c);
        for (int i = 0; i < q; ++i) {
            const double VW_a = VW * a[i];
            for (int c = 0; c < nb; ++c) b[i + c * q] = std::fma(VW_a, f[c], b[i + c * q]);
            for (int j = 0; j <= i; ++j) M[j + i * q] = std::fma(VW_a, a[j], M[j + i * q]);
        }
    });
    for (int i = 0; i < q - 1; ++i)
        for (int j = i + 1; j < q; ++j) M[j + i * q] = M[i + j * q];
    *info = 0;
    if (num_neighbors >= q) {
        *info = gepp_solve(q, nb, M, b);
        for (int c = 0; c < nb; ++c) out[c] = b[c * q];
    } else {
        for (int c = 0; c < nb; ++c) out[c] = 0.0;
    }
    return num_neighbors;
}

// ---------------------------------------------------------------------------------
// Post-processing LS type-B interpolation (analysis/common/lssph_b.py:21-143): value and
// first derivatives of one field at arbitrary points from every particle within h_eff.
// ---------------------------------------------------------------------------------
// Basis size of the post-processing interpolation (lssph_b.py:45-55).
int lsb_post_q(int sph_model, int target_problem) {
    const bool t4 = target_problem == 4;
    if (sph_model <= 3) return t4 ? 6 : 3;
    if (sph_model == 4) return t4 ? 10 : 6;
    if (sph_model == 5) return t4 ? 15 : 10;
    return t4 ? 21 : 15;
}

// Its basis columns on normalised offsets (lssph_b.py:83-125; the q = 6 / 10 orders differ
// from the q = 15 / 21 ones, as in the reference).
void lsb_post_basis(int q, double X, double Y, double* a) {
    a[0] = 1.0;
    a[1] = X;
    a[2] = Y;
    if (q == 3) return;
    const double X2 = X * X, Y2 = Y * Y;
    if (q == 6 || q == 10) {
        a[3] = 0.5 * X2;
        a[4] = X * Y;
        a[5] = 0.5 * Y2;
        if (q == 10) {
            a[6] = (1.0 / 6.0) * (X2 * X);
            a[7] = (0.5 * X2) * Y;
            a[8] = (0.5 * X) * Y2;
            a[9] = (1.0 / 6.0) * (Y2 * Y);
        }
        return;
    }
    const double X3 = X2 * X, Y3 = Y2 * Y, X4 = X2 * X2, Y4 = Y2 * Y2;
    a[3] = 0.5 * X2;
    a[4] = 0.5 * Y2;
    a[5] = X * Y;
    a[6] = (1.0 / 6.0) * X3;
    a[7] = (1.0 / 6.0) * Y3;
    a[8] = (0.5 * X2) * Y;
    a[9] = (0.5 * Y2) * X;
    a[10] = (1.0 / 24.0) * X4;
    a[11] = (1.0 / 24.0) * Y4;
    a[12] = ((1.0 / 6.0) * X3) * Y;
    a[13] = ((1.0 / 6.0) * Y3) * X;
    a[14] = (0.25 * X2) * Y2;
    if (q == 15) return;
    a[15] = (1.0 / 120.0) * (X4 * X);
    a[16] = (1.0 / 120.0) * (Y4 * Y);
    a[17] = ((1.0 / 24.0) * X4) * Y;
    a[18] = ((1.0 / 24.0) * Y4) * X;
    a[19] = ((1.0 / 12.0) * X3) * Y2;
    a[20] = ((1.0 / 12.0) * Y3) * X2;
}

// One target: neighbours in ascending particle index (the reference's sorted ball query),
// normal equations M = A^T W A, b = A^T W f with W = diag(W_ij V_j), GEPP.  NaN when fewer
// than q neighbours or a zero pivot (numpy's LinAlgError).  out = d0, d1 / h, d2 / h.
void lsb_post_point(const lssph_params& p, int q, double tx, double ty, const std::vector<int>& nbrs,
                    const double* X, const double* Y, const double* val, const double* rho, double* out) {
    const double h = p.h;
    if ((int)nbrs.size() < q) { out[0] = out[1] = out[2] = NAN; return; }
    double M[441] = {0}, b[21] = {0}, a[21];
    for (int j : nbrs) {
        const double dx = X[j] - tx, dy = Y[j] - ty;
        const double r = std::sqrt(dx * dx + dy * dy);
        const double w = cal_W(p.kernel_type, r, h) * (p.SP_mass / rho[j]);
        lsb_post_basis(q, dx / h, dy / h, a);
        for (int i = 0; i < q; ++i) {
            const double wa = w * a[i];
            b[i] = std::fma(wa, val[j], b[i]);
            for (int k = 0; k <= i; ++k) M[k + i * q] = std::fma(wa, a[k], M[k + i * q]);
        }
    }
    for (int i = 0; i < q - 1; ++i)
        for (int k = i + 1; k < q; ++k) M[k + i * q] = M[i + k * q];
    if (gepp_solve(q, 1, M, b) != 0) { out[0] = out[1] = out[2] = NAN; return; }
    out[0] = b[0];
    out[1] = b[1] / h;
    out[2] = b[2] / h;
}

// interpolate_LSSPH_B_mod.f90:24-178 (WALL_MODEL 2: q=3, 3: q=6)
void interpolate_LSSPH_B(orc_state* s, int me) {
    const lssph_params& p = s->p;
    const int q = (p.wall_model == 3) ? 6 : 3;
    const int nb = s->has_tem ? 4 : 3;
    double out[4];
    int info = 0;
    lssph_b_point(p, q, nb, s->vm_x[me], s->vm_y[me],
                  [&](auto&& f) {
                      for_candidates(s, s->idx_VM[me], [&](int you, double, double) {
                          if (s->ptype[you] == 0) f(you);
                      });
                  },
                  s->x.data(), s->y.data(), s->rho.data(),
                  [&](int you, int c) {
                      return c == 0 ? s->u[you] : c == 1 ? s->v[you] : c == 2 ? s->pre[you] : s->tem[you];
                  },
                  out, &info);
    if (info != 0) set_err(s, LSSPH_E_SINGULAR, "interpolate_LSSPH_B: singular moment matrix");
    s->vm_u[me] = out[0]; s->vm_v[me] = out[1]; s->vm_pre[me] = out[2];
    if (nb == 4) s->vm_tem[me] = out[3];
}

// interpolate_CSPH_mod.f90:24-130 (WALL_MODEL 1)
void interpolate_CSPH(orc_state* s, int me) {
    const lssph_params& p = s->p;
    const double h = p.h, h_eff_sq = p.h_eff * p.h_eff, SP_mass = p.SP_mass;
    const double my_x = s->vm_x[me], my_y = s->vm_y[me];
    double u = 0, v = 0, pre = 0, tem = 0, sw = 0;
    int num_neighbors = 0;
    for_candidates(s, s->idx_VM[me], [&](int you, double, double) {
        if (s->ptype[you] != 0) return;
        const double x_ij = my_x - s->x[you], y_ij = my_y - s->y[you];
        const double r2 = x_ij * x_ij + y_ij * y_ij;
        if (r2 > h_eff_sq) return;
        const double r = std::sqrt(r2);
        const double W = cal_W(p.kernel_type, r, h);
        ++num_neighbors;
        const double VW = (SP_mass / s->rho[you]) * W;
        sw = sw + VW;
        u = std::fma(VW, s->u[you], u);
        v = std::fma(VW, s->v[you], v);
        pre = std::fma(VW, s->pre[you], pre);
        if (s->has_tem) tem = std::fma(VW, s->tem[you], tem);
    });
    if (num_neighbors > 0 && sw > 1.0e-12) {
        s->vm_u[me] = u / sw; s->vm_v[me] = v / sw; s->vm_pre[me] = pre / sw;
        if (s->has_tem) s->vm_tem[me] = tem / sw;
    } else {
        s->vm_u[me] = 0.0; s->vm_v[me] = 0.0; s->vm_pre[me] = 0.0;
        if (s->has_tem) s->vm_tem[me] = 0.0;
    }
}

// extrapolate_VM_to_WL_mod.f90:23-275
void extrapolate_VM_to_WL(orc_state* s, int me) {
    const lssph_params& p = s->p;
    const int you = s->vm_pair[me];
    const double nx = s->vm_nx[me], ny = s->vm_ny[me];
    const double vu = s->vm_u[me], vv = s->vm_v[me], vp = s->vm_pre[me], vt = s->vm_tem[me];
    const bool P4 = p.target_problem == 4;
    auto velocity = [&](int bc) {
        if (bc == 1) {
            const double u_n = vu * nx + vv * ny;
            s->u[you] = vu - (2.0 * u_n) * nx;
            s->v[you] = vv - (2.0 * u_n) * ny;
        } else if (bc == 2) {
            s->u[you] = -vu; s->v[you] = -vv;
        } else if (bc == 3) {
            s->u[you] = 2.0 * p.u_top - vu; s->v[you] = -vv;
        }
    };
    auto hydro = [&](int tbc, double Tw) {
        if (P4 && tbc == 1)
            s->pre[you] = vp + (((p.rho_ref * p.alpha_ref) * (Tw - p.tem_ave)) * p.gravity) * (s->y[you] - s->vm_y[me]);
        else
            s->pre[you] = vp;
    };
    auto temp = [&](int tbc, double Tw) {
        if (!P4) return;
        if (tbc == 1) s->tem[you] = 2.0 * Tw - vt;
        else if (tbc == 2) s->tem[you] = vt;
    };
    switch (s->vm_ptype[me]) {
        case 1: velocity(p.u_bc_bottom); hydro(p.tem_bc_bottom, p.tem_bottom); temp(p.tem_bc_bottom, p.tem_bottom); break;
        case 2: velocity(p.u_bc_top); hydro(p.tem_bc_top, p.tem_top); temp(p.tem_bc_top, p.tem_top); break;
        case 3: velocity(p.u_bc_left); s->pre[you] = vp; temp(p.tem_bc_left, p.tem_left); break;
        case 4: velocity(p.u_bc_right); s->pre[you] = vp; temp(p.tem_bc_right, p.tem_right); break;
        case 5: case 6:
            s->u[you] = -vu; s->v[you] = -vv;
            hydro(p.tem_bc_bottom, p.tem_bottom); temp(p.tem_bc_bottom, p.tem_bottom); break;
        case 7: case 8:
            if (p.u_bc_top == 3) { s->u[you] = 2.0 * p.u_top - vu; s->v[you] = -vv; }
            else { s->u[you] = -vu; s->v[you] = -vv; }
            hydro(p.tem_bc_top, p.tem_top); temp(p.tem_bc_top, p.tem_top); break;
        default: break;
    }
}

// extrapolate_diff_test_mod.f90:24-106
void extrapolate_diff_test(orc_state* s, int me) {
    const lssph_params& p = s->p;
    const int you = s->vm_pair[me];
    const double vu = s->vm_u[me];
    switch (s->vm_ptype[me]) {
        case 1:
            if (p.u_bc_bottom == 1) s->u[you] = vu;
            else if (p.u_bc_bottom == 2) s->u[you] = 2.0 * std::sin(PI * (s->vm_x[me] - p.WL_thick)) - vu;
            break;
        case 2:
            if (p.u_bc_top == 1) s->u[you] = vu;
            else if (p.u_bc_top == 2) s->u[you] = 2.0 * (-std::sin(PI * (s->vm_x[me] - p.WL_thick))) - vu;
            break;
        case 3:
            if (p.u_bc_left == 1)
                s->u[you] = vu + (PI * std::cos(PI * (s->vm_y[me] - p.WL_thick))) * (s->x[you] - s->vm_x[me]);
            else if (p.u_bc_left == 2) s->u[you] = -vu;
            break;
        case 4:
            if (p.u_bc_right == 1)
                s->u[you] = vu + ((-PI) * std::cos(PI * (s->vm_y[me] - p.WL_thick))) * (s->x[you] - s->vm_x[me]);
            else if (p.u_bc_right == 2) s->u[you] = -vu;
            break;
        case 5: case 6: case 7: case 8: s->u[you] = -vu; break;
        default: break;
    }
}

// ghost_mod.f90:43-78
void ghost(orc_state* s) {
    const int ne = s->num_ext;
    const int wm = s->p.wall_model;
    const bool diff = s->p.target_problem == 1;
#pragma omp parallel for schedule(static)
    for (int me = 0; me < ne; ++me) {
        if (wm == 1) interpolate_CSPH(s, me);
        else interpolate_LSSPH_B(s, me);
        if (diff) extrapolate_diff_test(s, me);
        else extrapolate_VM_to_WL(s, me);
    }
}

// RK2_mod.f90:30-128
void RK2(orc_state* s) {
    const lssph_params& p = s->p;
    const int n = s->num_int;
    const double c_sq = p.sound_speed * p.sound_speed, rho_ref = p.rho_ref;
    const bool P1 = p.target_problem == 1;
#pragma omp parallel for schedule(static)
    for (int me = 0; me < n; ++me) {
        s->x_old[me] = s->x[me]; s->y_old[me] = s->y[me]; s->u_old[me] = s->u[me];
        s->v_old[me] = s->v[me]; s->rho_old[me] = s->rho[me];
        if (s->has_tem) s->tem_old[me] = s->tem[me];
    }
    for (int st = 1; st <= 2; ++st) {
        calculate_RHS(s);
        const double dt_eff = (st == 1) ? p.dt / 2.0 : p.dt;
#pragma omp parallel for schedule(static)
        for (int me = 0; me < n; ++me) {
            if (!P1) {
                s->x[me] = s->x_old[me] + s->u[me] * dt_eff;
                s->y[me] = s->y_old[me] + s->v[me] * dt_eff;
                if (p.periodic) { s->x[me] = wrap_pos(s->x[me], p.len_x); s->y[me] = wrap_pos(s->y[me], p.len_y); }
                s->v[me] = s->v_old[me] + s->RHS_v[me] * dt_eff;
                s->rho[me] = s->rho_old[me] + s->RHS_rho[me] * dt_eff;
            }
            s->u[me] = s->u_old[me] + s->RHS_u[me] * dt_eff;
            if (s->has_tem) s->tem[me] = s->tem_old[me] + s->RHS_tem[me] * dt_eff;
            if (!P1) s->pre[me] = c_sq * (s->rho[me] - rho_ref);
        }
        if (!P1) update_cell(s);
        ghost(s);
    }
}

// RK4_mod.f90:30-179
void RK4(orc_state* s) {
    const lssph_params& p = s->p;
    const int n = s->num_int;
    const double c_sq = p.sound_speed * p.sound_speed, rho_ref = p.rho_ref;
    const bool P1 = p.target_problem == 1;
#pragma omp parallel for schedule(static)
    for (int me = 0; me < n; ++me) {
        s->x_old[me] = s->x[me]; s->y_old[me] = s->y[me]; s->u_old[me] = s->u[me];
        s->v_old[me] = s->v[me]; s->rho_old[me] = s->rho[me];
        if (s->has_tem) s->tem_old[me] = s->tem[me];
        s->x_new[me] = s->x[me]; s->y_new[me] = s->y[me]; s->u_new[me] = s->u[me];
        s->v_new[me] = s->v[me]; s->rho_new[me] = s->rho[me];
        if (s->has_tem) s->tem_new[me] = s->tem[me];
    }
    for (int st = 1; st <= 4; ++st) {
        calculate_RHS(s);
        double dt_1, dt_2;
        if (st == 1) { dt_1 = p.dt / 6.0; dt_2 = p.dt / 2.0; }
        else if (st == 2) { dt_1 = p.dt / 3.0; dt_2 = p.dt / 2.0; }
        else if (st == 3) { dt_1 = p.dt / 3.0; dt_2 = p.dt; }
        else { dt_1 = p.dt / 6.0; dt_2 = 0.0; }
#pragma omp parallel for schedule(static)
        for (int me = 0; me < n; ++me) {
            s->u_new[me] = s->u_new[me] + s->RHS_u[me] * dt_1;
            if (!P1) {
                s->v_new[me] = s->v_new[me] + s->RHS_v[me] * dt_1;
                s->x_new[me] = s->x_new[me] + s->u[me] * dt_1;
                s->y_new[me] = s->y_new[me] + s->v[me] * dt_1;
                s->rho_new[me] = s->rho_new[me] + s->RHS_rho[me] * dt_1;
            }
            if (s->has_tem) s->tem_new[me] = s->tem_new[me] + s->RHS_tem[me] * dt_1;
            if (st < 4) {
                if (!P1) {
                    s->x[me] = s->x_old[me] + s->u[me] * dt_2;
                    s->y[me] = s->y_old[me] + s->v[me] * dt_2;
                    if (p.periodic) { s->x[me] = wrap_pos(s->x[me], p.len_x); s->y[me] = wrap_pos(s->y[me], p.len_y); }
                    s->v[me] = s->v_old[me] + s->RHS_v[me] * dt_2;
                    s->rho[me] = s->rho_old[me] + s->RHS_rho[me] * dt_2;
                }
                s->u[me] = s->u_old[me] + s->RHS_u[me] * dt_2;
                if (s->has_tem) s->tem[me] = s->tem_old[me] + s->RHS_tem[me] * dt_2;
            } else {
                s->u[me] = s->u_new[me];
                if (!P1) {
                    s->v[me] = s->v_new[me]; s->x[me] = s->x_new[me]; s->y[me] = s->y_new[me];
                    s->rho[me] = s->rho_new[me];
                    if (p.periodic) { s->x[me] = wrap_pos(s->x[me], p.len_x); s->y[me] = wrap_pos(s->y[me], p.len_y); }
                }
                if (s->has_tem) s->tem[me] = s->tem_new[me];
            }
            if (!P1) s->pre[me] = c_sq * (s->rho[me] - rho_ref);
        }
        if (!P1) update_cell(s);
        ghost(s);
    }
}

// shift_interpolate_mod.f90:23-300
void shift_interpolate(orc_state* s, int me, double coe_PST) {
    const lssph_params& p = s->p;
    const int k = (p.sph_model <= 2) ? 1 : order_of_model(p.sph_model);
    const int q = (k == 1) ? 2 : (k == 2) ? 5 : (k == 3) ? 9 : (k == 4) ? 14 : 20;
    const int nb = s->has_tem ? 4 : 3;
    const double h = p.h, h_eff_sq = p.h_eff * p.h_eff, SP_mass = p.SP_mass, W_ave = p.W_ave;
    double ih[5];
    ih[0] = 1.0 / h;
    for (int i = 1; i < k; ++i) ih[i] = ih[i - 1] / h;
    const double my_x = s->x[me], my_y = s->y[me], my_u = s->u[me], my_v = s->v[me], my_rho = s->rho[me];
    const double my_tem = s->has_tem ? s->tem[me] : 0.0;
    double M[400] = {0}, b[80] = {0}, a[20] = {0};
    double dx = 0.0, dy = 0.0;
    int num_neighbors = 0;
    for_candidates(s, s->idx_SP[me], [&](int you, double sx, double sy) {
        if (me == you) return;
        const double x_ji = (s->x[you] + sx) - my_x, y_ji = (s->y[you] + sy) - my_y;
        const double r2 = x_ji * x_ji + y_ji * y_ji;
        if (r2 > h_eff_sq) return;
        const double r = std::sqrt(r2);
        const double W = cal_W(p.kernel_type, r, h);
        const double dW_dr = cal_dW(p.kernel_type, r, h);
        ++num_neighbors;
        const double V_j = SP_mass / s->rho[you];
        const double VW = V_j * W;
        const double rinv = 1.0 / r;
        const double gx = ((dW_dr * (-x_ji)) * rinv) * V_j;
        const double gy = ((dW_dr * (-y_ji)) * rinv) * V_j;
        const double t = W * (1.0 / W_ave), t2 = t * t, t4 = t2 * t2;
        const double fac = 1.0 + 0.2 * t4;
        dx = std::fma(fac, gx, dx);
        dy = std::fma(fac, gy, dy);
        basis_A(k, x_ji, y_ji, ih, a);
        double df[4] = {s->u[you] - my_u, s->v[you] - my_v, s->rho[you] - my_rho,
                        nb == 4 ? s->tem[you] - my_tem : 0.0};
        for (int i = 0; i < q; ++i) {
            const double VW_a = VW * a[i];
            for (int c = 0; c < nb; ++c) b[i + c * q] = std::fma(VW_a, df[c], b[i + c * q]);
            for (int j = 0; j <= i; ++j) M[j + i * q] = std::fma(VW_a, a[j], M[j + i * q]);
        }
    });
    dx = -coe_PST * dx;
    dy = -coe_PST * dy;
    const double rr = std::sqrt(dx * dx + dy * dy);
    if (rr > 0.2 * h) {
        dx = ((0.2 * h) * dx) / rr;
        dy = ((0.2 * h) * dy) / rr;
    }
    s->x_old[me] = s->x[me] + dx;
    s->y_old[me] = s->y[me] + dy;
    for (int i = 0; i < q - 1; ++i)
        for (int j = i + 1; j < q; ++j) M[j + i * q] = M[i + j * q];
    if (num_neighbors >= q) {
        if (gepp_solve(q, nb, M, b) != 0) set_err(s, LSSPH_E_SINGULAR, "shift_interpolate: singular moment matrix");
    } else {
        std::fill(b, b + 80, 0.0);
    }
    basis_A(k, dx, dy, ih, a);
    double acc[4];
    for (int c = 0; c < nb; ++c) {
        double sacc = 0.0;
        for (int i = 0; i < q; ++i) sacc = std::fma(a[i], b[i + c * q], sacc);
        acc[c] = sacc;
    }
    s->u_old[me] = s->u[me] + acc[0];
    s->v_old[me] = s->v[me] + acc[1];
    s->rho_old[me] = s->rho[me] + acc[2];
    if (nb == 4) s->tem_old[me] = s->tem[me] + acc[3];
}

// PST_mod.f90:28-116
void PST(orc_state* s) {
    const lssph_params& p = s->p;
    const int n = s->num_int;
    const double c_sq = p.sound_speed * p.sound_speed, rho_ref = p.rho_ref;
    double U_max = 0.0;
#pragma omp parallel for reduction(max : U_max) schedule(static)
    for (int me = 0; me < n; ++me) {
        const double U = std::sqrt(s->u[me] * s->u[me] + s->v[me] * s->v[me]);
        U_max = std::max(U_max, U);
    }
    const double coe_PST = ((p.PST_c * U_max) * p.dt) * p.h;
#pragma omp parallel for schedule(static)
    for (int me = 0; me < n; ++me) shift_interpolate(s, me, coe_PST);
#pragma omp parallel for schedule(static)
    for (int me = 0; me < n; ++me) {
        s->x[me] = s->x_old[me]; s->y[me] = s->y_old[me]; s->u[me] = s->u_old[me];
        s->v[me] = s->v_old[me]; s->rho[me] = s->rho_old[me];
        if (p.periodic) { s->x[me] = wrap_pos(s->x[me], p.len_x); s->y[me] = wrap_pos(s->y[me], p.len_y); }
        if (s->has_tem) s->tem[me] = s->tem_old[me];
        s->pre[me] = c_sq * (s->rho[me] - rho_ref);
    }
    if (p.target_problem != 1) update_cell(s);
    ghost(s);
}

// check_steady_state_mod.f90:23-69
int check_steady_state(orc_state* s) {
    const int n = s->num_int;
    double df_max = 0.0;
#pragma omp parallel for reduction(max : df_max) schedule(static)
    for (int me = 0; me < n; ++me) df_max = std::max(std::fabs(s->f_previous[me] - s->u[me]), df_max);
    if (df_max < s->p.threshold) return 1;
#pragma omp parallel for schedule(static)
    for (int me = 0; me < n; ++me) s->f_previous[me] = s->u[me];
    return 0;
}

// Time-loop body (main.f90:119-149); returns the steady step (1-based in this call) or 0.
int run_steps(orc_state* s, int nsteps) {
    for (int st = 1; st <= nsteps; ++st) {
        if (s->p.rk == 2) RK2(s); else RK4(s);
        if (s->p.target_problem != 1) PST(s);
        if (s->p.target_problem == 1 && check_steady_state(s)) return st;
    }
    return 0;
}

void copy_out(const std::vector<double>& v, double* dst, int n) {
    if (dst) std::memcpy(dst, v.data(), sizeof(double) * (size_t)n);
}

}  // namespace

// =====================================================================================
// extern "C" API used by tests/ (ctypes) and bench.py's CPU baseline.
// =====================================================================================
extern "C" {

const char* orc_last_error(void) { return g_err.c_str(); }

int orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

int orc_init_param(lssph_params* p) { init_param(p); return 0; }

size_t orc_params_sizeof(void) { return sizeof(lssph_params); }

// The reference's shipped config.h (config.h:24-200: TARGET_PROBLEM 2 ... WALL_MODEL 2),
// then init_param, so that the oracle builds its parameters without the engine library.
// precision / lanes / seed / periodic are engine-side extensions and start at zero.
int orc_params_default(lssph_params* p) {
    std::memset(p, 0, sizeof(*p));
    p->target_problem = 2;                                            // config.h:24
    p->u_bc_top = 1; p->u_bc_bottom = 1; p->u_bc_left = 1; p->u_bc_right = 1;   // :35-38
    p->u_top = 1.0;                                                   // :42
    p->tem_bc_top = 1; p->tem_bc_bottom = 1; p->tem_bc_left = 2; p->tem_bc_right = 2;  // :52-55
    p->tem_top = 0.0; p->tem_bottom = 1.0e-2; p->tem_left = 0.0; p->tem_right = 0.0;  // :59-62
    std::snprintf(p->save_name, sizeof(p->save_name), "%s", "tg_compare_100_write");  // :69
    std::snprintf(p->read_name, sizeof(p->read_name), "%s", "new");                   // :72
    p->omp_threads = 8;                                               // :79
    p->len_x = 1.0; p->len_y = 1.0;                                   // :86-87
    p->num_x = 100; p->num_y = 100;                                   // :91-92
    p->rk = 4;                                                        // :99
    p->start_step = 1; p->end_step = 10000; p->write_step = 100;      // :103-109
    p->threshold = 1.0e-10;                                           // :112
    p->coe_CFL = 0.5; p->coe_dif = 0.2;                               // :117-118
    p->zeta_RSST = 1.0; p->xi_VIM = 1.0;                              // :123-124
    p->rho_ref = 1.0; p->vis_ref = 1.0e-2; p->K_ref = 1.0e2;          // :131-137
    p->k_th_ref = 1.0e-2; p->cp_ref = 1.0e3; p->alpha_ref = 7.1e-3;   // :140-146
    p->gravity = 10.0; p->pos_pert = 0.0;                             // :152-155
    p->tg_a = 1; p->tg_b = 1;                                         // :158-159
    p->coe_h = 1.2; p->PST_c = 1.5; p->coe_delta_sph = 0.0;           // :166-175
    p->kernel_type = 3; p->sph_model = 3; p->wall_model = 2;          // :188-213
    init_param(p);
    return 0;
}

double orc_kernel_W(int kt, double r, double h) { return cal_W(kt, r, h); }
double orc_kernel_dW(int kt, double r, double h) { return cal_dW(kt, r, h); }

// n x n column-major A, n x nrhs column-major B (solution overwrites B).  Returns INFO.
int orc_dgesv(int n, int nrhs, double* A, double* B) { return gepp_solve(n, nrhs, A, B); }

// Fresh start: setup_closed_box + impose_* + init_virtual_markers + init_cell +
// update_cell, then (do_ghost = 1) ghost as the write_param call does
// (write_param_mod.f90:144).
orc_state* orc_create_new(const lssph_params* p, int do_ghost) {
    orc_state* s = new orc_state();
    s->p = *p;
    s->has_tem = p->target_problem == 4;
    setup_closed_box(s);
    impose_ic(s);
    alloc_work(s);
    init_virtual_markers(s);
    init_cell(s);
    update_cell(s);
    if (do_ghost) ghost(s);
    return s;
}

// Start from given state (all num_total particles, reference order), e.g. a restart file
// or positions shared with the engine.  do_ghost = 1 runs ghost() after the cell build.
orc_state* orc_create_from(const lssph_params* p, int num_total, int num_int, const int32_t* ptype,
                           const double* x, const double* y, const double* u, const double* v,
                           const double* rho, const double* pre, const double* tem, int do_ghost) {
    orc_state* s = new orc_state();
    s->p = *p;
    s->has_tem = p->target_problem == 4;
    s->num_total = num_total;
    s->num_int = num_int;
    s->num_ext = num_total - num_int;
    s->ptype.assign(ptype, ptype + num_total);
    s->x.assign(x, x + num_total); s->y.assign(y, y + num_total);
    s->u.assign(u, u + num_total); s->v.assign(v, v + num_total);
    s->rho.assign(rho, rho + num_total); s->pre.assign(pre, pre + num_total);
    if (tem) s->tem.assign(tem, tem + num_total); else s->tem.assign(num_total, 0.0);
    alloc_work(s);
    init_virtual_markers(s);
    init_cell(s);
    update_cell(s);
    if (do_ghost) ghost(s);
    return s;
}

void orc_destroy(orc_state* s) { delete s; }

int orc_error(const orc_state* s) { return s->error; }

int orc_sizes(const orc_state* s, int* num_total, int* num_int, int* num_ext, int* ncell, int* list_cap) {
    if (num_total) *num_total = s->num_total;
    if (num_int) *num_int = s->num_int;
    if (num_ext) *num_ext = s->num_ext;
    if (ncell) *ncell = s->idx_max;
    if (list_cap) *list_cap = s->list_cap;
    return 0;
}

int orc_get(const orc_state* s, int32_t* ptype, double* x, double* y, double* u, double* v,
            double* rho, double* pre, double* tem) {
    const int n = s->num_total;
    if (ptype) std::memcpy(ptype, s->ptype.data(), sizeof(int32_t) * (size_t)n);
    copy_out(s->x, x, n); copy_out(s->y, y, n); copy_out(s->u, u, n); copy_out(s->v, v, n);
    copy_out(s->rho, rho, n); copy_out(s->pre, pre, n); copy_out(s->tem, tem, n);
    return 0;
}

int orc_set(orc_state* s, const double* x, const double* y, const double* u, const double* v,
            const double* rho, const double* pre, const double* tem) {
    const int n = s->num_total;
    if (x) s->x.assign(x, x + n);
    if (y) s->y.assign(y, y + n);
    if (u) s->u.assign(u, u + n);
    if (v) s->v.assign(v, v + n);
    if (rho) s->rho.assign(rho, rho + n);
    if (pre) s->pre.assign(pre, pre + n);
    if (tem) s->tem.assign(tem, tem + n);
    return 0;
}

int orc_get_rhs(const orc_state* s, double* ru, double* rv, double* rr, double* rt) {
    const int n = s->num_int;
    copy_out(s->RHS_u, ru, n); copy_out(s->RHS_v, rv, n); copy_out(s->RHS_rho, rr, n);
    copy_out(s->RHS_tem, rt, n);
    return 0;
}

int orc_get_vm(const orc_state* s, int32_t* ptype, double* x, double* y, double* u, double* v,
               double* pre, double* tem, double* nx, double* ny) {
    const int n = s->num_ext;
    if (ptype) std::memcpy(ptype, s->vm_ptype.data(), sizeof(int32_t) * (size_t)n);
    copy_out(s->vm_x, x, n); copy_out(s->vm_y, y, n); copy_out(s->vm_u, u, n);
    copy_out(s->vm_v, v, n); copy_out(s->vm_pre, pre, n); copy_out(s->vm_tem, tem, n);
    copy_out(s->vm_nx, nx, n); copy_out(s->vm_ny, ny, n);
    return 0;
}

int orc_get_cells(const orc_state* s, int32_t* idx_SP, int32_t* idx_VM) {
    if (idx_SP) std::memcpy(idx_SP, s->idx_SP.data(), sizeof(int32_t) * (size_t)s->num_total);
    if (idx_VM) std::memcpy(idx_VM, s->idx_VM.data(), sizeof(int32_t) * (size_t)s->num_ext);
    return 0;
}

// LS type-B interpolation of one field at target points over a particle cloud, brute-force
// candidates in index order (the math of interpolate_LSSPH_B_mod.f90 / lssph_b.py:55-140).
// p supplies h, h_eff, SP_mass, kernel_type.  Returns the number of targets with < q
// neighbours (their output is 0).
int orc_lssph_b(const lssph_params* p, int q, int n_src, const double* xs, const double* ys, const double* rho,
                const double* val, int n_tgt, const double* xt, const double* yt, double* out) {
    int short_count = 0;
    for (int t = 0; t < n_tgt; ++t) {
        double o[1];
        int info = 0;
        const int nn = lssph_b_point(*p, q, 1, xt[t], yt[t],
                                     [&](auto&& f) { for (int j = 0; j < n_src; ++j) f(j); },
                                     xs, ys, rho, [&](int you, int) { return val[you]; }, o, &info);
        if (nn < q) ++short_count;
        out[t] = o[0];
    }
    return short_count;
}

// analysis/common/lssph_b.py:21-143 over n_src particles at n_tgt points; out[3 * t + k].
// The ball query bins the particles into cells of h_eff and sorts each target's hits by
// index, which gives the same neighbour list as the reference's KD-tree query.
int orc_lsb_post(const lssph_params* p, int n_src, const double* xs, const double* ys, const double* val,
                 const double* rho, int n_tgt, const double* xt, const double* yt, double* out) {
    const int q = lsb_post_q(p->sph_model, p->target_problem);
    if (n_src <= 0) {
        for (int t = 0; t < 3 * n_tgt; ++t) out[t] = NAN;
        return q;
    }
    const double he = p->h_eff, he2 = he * he;
    double x0 = xs[0], y0 = ys[0], x1 = xs[0], y1 = ys[0];
    for (int j = 1; j < n_src; ++j) {
        x0 = std::min(x0, xs[j]); x1 = std::max(x1, xs[j]);
        y0 = std::min(y0, ys[j]); y1 = std::max(y1, ys[j]);
    }
    const int ncx = (int)std::floor((x1 - x0) / he) + 1, ncy = (int)std::floor((y1 - y0) / he) + 1;
    std::vector<std::vector<int>> cells((size_t)ncx * ncy);
    for (int j = 0; j < n_src; ++j) {
        const int cx = std::min(ncx - 1, (int)std::floor((xs[j] - x0) / he));
        const int cy = std::min(ncy - 1, (int)std::floor((ys[j] - y0) / he));
        cells[(size_t)cy * ncx + cx].push_back(j);
    }
#pragma omp parallel for schedule(dynamic, 16)
    for (int t = 0; t < n_tgt; ++t) {
        std::vector<int> nb;
        const double fx = std::floor((xt[t] - x0) / he), fy = std::floor((yt[t] - y0) / he);
        if (fx >= -1.0 && fx <= ncx && fy >= -1.0 && fy <= ncy) {
            const int cx = (int)fx, cy = (int)fy;
            for (int yy = std::max(cy - 1, 0); yy <= std::min(cy + 1, ncy - 1); ++yy)
                for (int xx = std::max(cx - 1, 0); xx <= std::min(cx + 1, ncx - 1); ++xx)
                    for (int j : cells[(size_t)yy * ncx + xx]) {
                        const double dx = xs[j] - xt[t], dy = ys[j] - yt[t];
                        if (dx * dx + dy * dy <= he2) nb.push_back(j);
                    }
        }
        std::sort(nb.begin(), nb.end());
        lsb_post_point(*p, q, xt[t], yt[t], nb, xs, ys, val, rho, out + 3 * t);
    }
    return q;
}

int orc_calculate_rhs(orc_state* s) { calculate_RHS(s); return s->error; }
int orc_update_cell(orc_state* s) { update_cell(s); return s->error; }
int orc_ghost(orc_state* s) { ghost(s); return s->error; }
int orc_rk2(orc_state* s) { RK2(s); return s->error; }
int orc_rk4(orc_state* s) { RK4(s); return s->error; }
int orc_pst(orc_state* s) { PST(s); return s->error; }
int orc_check_steady_state(orc_state* s, int* is_steady) { *is_steady = check_steady_state(s); return 0; }
int orc_run(orc_state* s, int nsteps, int* steady_step) {
    const int st = run_steps(s, nsteps);
    if (steady_step) *steady_step = st;
    return s->error;
}

// Sorted in-radius neighbour sets.  which = 0: interior particles over all candidates
// (LSSPH_A_mod.f90:102-125); which = 1: virtual markers over fluid candidates
// (interpolate_LSSPH_B_mod.f90:158-180).  offsets has n+1 entries.  Returns nnz or -1.
int64_t orc_neighbors_csr(const orc_state* s, int which, int32_t* offsets, int32_t* idx, int64_t cap) {
    const double h_eff_sq = s->p.h_eff * s->p.h_eff;
    const int n = which == 0 ? s->num_int : s->num_ext;
    int64_t nnz = 0;
    std::vector<int> tmp;
    for (int me = 0; me < n; ++me) {
        offsets[me] = (int32_t)nnz;
        tmp.clear();
        const double mx = which == 0 ? s->x[me] : s->vm_x[me];
        const double my = which == 0 ? s->y[me] : s->vm_y[me];
        const int cell = which == 0 ? s->idx_SP[me] : s->idx_VM[me];
        for_candidates(s, cell, [&](int you, double sx, double sy) {
            if (which == 0 && you == me) return;
            if (which == 1 && s->ptype[you] != 0) return;
            const double xj = (s->x[you] + sx) - mx, yj = (s->y[you] + sy) - my;
            if (xj * xj + yj * yj > h_eff_sq) return;
            tmp.push_back(you);
        });
        std::sort(tmp.begin(), tmp.end());
        if (nnz + (int64_t)tmp.size() > cap) return -1;
        for (int t : tmp) idx[nnz++] = t;
    }
    offsets[n] = (int32_t)nnz;
    return nnz;
}

}  // extern "C"
