// kernels.cuh -- device code of the LS-SPH path (sm_100a): FP64, and a mixed-precision
// variant of the stage and PST kernels (FP32 pair phase, FP64 solve and RK update).
//
// Every kernel here replaces one OpenMP region of the reference solver:
//   k_stage      calculate_RHS (LSSPH_A_mod.f90:26-271) fused with the RK2/RK4 stage
//                update + EOS (RK2_mod.f90:87-108, RK4_mod.f90:109-159) and with the
//                scatter half of update_cell (update_cell_mod.f90:40-70)
//   k_ghost      ghost (ghost_mod.f90:55-74): LS type-B / CSPH interpolation at each
//                virtual marker + extrapolation to its ghost particle
//   k_pst        shift_interpolate (shift_interpolate_mod.f90:23-300) fused with the
//                PST copy-back + EOS (PST_mod.f90:85-99) and the cell scatter
// The cell lists are left in scatter (atomic) order; every consumer rebuilds the
// reference order of update_cell (interior particles by ascending index, then the static
// ghost list, update_cell_mod.f90:49-93) while staging a tile in shared memory.
//
// Work decomposition: one CTA per tile of TX x TY cells.  The CTA stages the particles of
// the (TX+2) x (TY+2) halo cells into shared memory with independent loads (all in
// flight at once), then each particle of the tile's own cells runs its neighbour loop
// out of shared memory: the 3x3 candidate cells of any own particle lie in the halo.
//
// Arithmetic follows the oracle's sequence: the file is compiled with -fmad=false so
// no multiply-add is fused implicitly, and fma() appears only at the accumulation sites
// and in the LU.  With one lane per particle the neighbour loop visits candidates in
// the reference list order and the results are bit-identical to the oracle; with G>1
// lanes each lane sums a strided share of the list and a butterfly shuffle combines the
// partial sums (identical on every lane, so the G lanes agree bit for bit).
#pragma once

#include <cstddef>
#include <type_traits>

#include <cuda_runtime.h>
#include <stdint.h>

namespace lssph {

// ---- error bits (device scalars) -----------------------------------------------------
enum : int {
    ERR_CELL_OVERFLOW = 1,
    ERR_OUT_OF_DOMAIN = 2,
    ERR_NONFINITE = 4,
};
enum : int { WARN_SINGULAR = 1 };

struct Scalars {
    unsigned long long umax2;   // max(u^2+v^2) bits (non-negative doubles order as uint64)
    unsigned long long dfmax;   // max |f_previous - u| bits (problem 1)
    int err;                    // ERR_* bits; any set bit halts later kernels
    int warn;                   // WARN_* bits
    int steady;                 // 1 once the steady state is reached (problem 1)
    int step_count;             // time steps completed
    int steady_step;            // step_count value at which steady was reached
    int step_limit;             // stop once step_count reaches it (0 = no budget)
    int done;                   // 1 once the step budget is used up
    int ctas_done;              // CTAs of the current end-of-step launch that have finished
    int step_mark;              // step_count at the start of the current lssph_step call
};
static_assert(offsetof(Scalars, done) == offsetof(Scalars, step_limit) + sizeof(int),
              "step_limit and done are written together");

// Constants of one solve (a subset of lssph_params plus precomputed factors).
struct Phys {
    int problem, kt, rk, wall_model;
    int u_bc_top, u_bc_bottom, u_bc_left, u_bc_right;
    int tem_bc_top, tem_bc_bottom, tem_bc_left, tem_bc_right;
    int nx, ny, ncell, cap;
    int num_total, num_int, num_ext, sph_model;
    int periodic;         // periodic: square domain (0, Lx]^2, cells wrap, no ghosts
    int split_pos;        // mixed precision: every position write also writes Fld::ox, oy
    double u_top, tem_top, tem_bottom, tem_left, tem_right;
    double h, ih1, ih2A, ih2B, h_eff_sq, inv_h_eff, SP_mass, W_ave, wnorm, dt;
    double c_sq, rho_ref, vis_ref, delta, zeta_sq, xi_sq, alpha_ref, gravity, tem_ave;
    double thermal_dif, PST_c, threshold, hydro_coef_top, hydro_coef_bottom;
    // reciprocals of loop-invariant divisors (1/W_ave, 1/zeta^2, 1/xi^2, -3/h, -5/h)
    double iWave, izeta2, ixi2, m3h, m5h;
    double Lx;   // periodic domain side
    double cw;   // cell width: the origin of cell (cx, cy) is (cx * cw, cy * cw)
};

// Periodic position wrap into (0, L] (the oracle's wrap_pos).
__device__ __forceinline__ double wrap_pos(double x, double L) { return x <= 0.0 ? x + L : (x > L ? x - L : x); }

struct Fld {   // SoA particle state over num_total
    double *x, *y, *u, *v, *rho, *pre, *tem, *vol;
    // Split-precision positions (mixed precision): the FP32 offset of each particle from the
    // FP64 origin of the cell that holds it, kept beside the FP64 positions of the RK update.
    float *ox, *oy;
};

// Split-precision position of particle i, held by cell `key`.
__device__ __forceinline__ void put_split_pos(const Phys& P, const Fld& F, int i, double x, double y, int key) {
    const int cx = key % P.nx, cy = key / P.nx;
    F.ox[i] = (float)(x - (double)cx * P.cw);
    F.oy[i] = (float)(y - (double)cy * P.cw);
}
// Cell lists rotate through three buffers: a stage reads list l and scatters into list
// l + 1 while the ghost launch after it clears list l - 1, so a list is cleared well
// before the next scatter into it and no clearing sits between two launches that read
// the same buffers.
constexpr int kLists = 3;
__host__ __device__ constexpr int next_list(int l) { return l == kLists - 1 ? 0 : l + 1; }
__host__ __device__ constexpr int prev_list(int l) { return l == 0 ? kLists - 1 : l - 1; }

struct Lst {   // interior particles per cell, scatter order: slots[c*cap + k], k < cnt[c]
    int *cnt, *slots;
};
struct Work {  // per-interior-particle arrays
    double *x_old, *y_old, *u_old, *v_old, *rho_old, *tem_old;
    double *x_acc, *y_acc, *u_acc, *v_acc, *rho_acc, *tem_acc;
    double *rhs_u, *rhs_v, *rhs_rho, *rhs_tem;
    double *f_prev, *src;
    int* key;
    // mixed precision, split shape: the reduced pair sums of every interior particle, entry e
    // of particle i at sums[e * num_int + i] (MXS_ENTRIES entries)
    double* sums;
};
struct VMd {   // virtual markers over num_ext
    double *x, *y, *nx, *ny, *u, *v, *pre, *tem, *K;
    int *ptype, *key, *mode;
};

enum : int { MODE_STAGE = 0, MODE_RHS_ONLY = 1 };
struct StageCfg {
    int mode;        // MODE_*
    int stage;       // 1-based RK stage
    int last;        // last stage of the step
    int do_scatter;  // rebuild the cell list of the new positions
    int do_umax;     // reduce max(u^2+v^2) of the new state for PST
    int do_steady;   // problem-1 steady-state reduction + f_previous copy
    int write_rhs;   // keep RHS arrays
    int pad;
    double dt1, dt2; // RK4: accumulator / intermediate factors; RK2: dt2 = dt_eff
};

// P1 ghost extrapolation modes (extrapolate_diff_test_mod.f90:40-103), K precomputed.
enum : int { XM_COPY = 0, XM_K_MINUS = 1, XM_PLUS_K = 2, XM_NEG = 3 };

// ---------------------------------------------------------------------------------------
// Programmatic dependent launch: a kernel launched with programmatic stream serialisation
// can be scheduled while its predecessor drains; pdl_wait() holds it until the predecessor
// has completed and its writes are visible, pdl_release() lets the successor be scheduled.
// Both are no-ops for an ordinary launch.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_release() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

__device__ __forceinline__ bool halted(const Scalars* sc) {
    return (*(volatile const int*)&sc->err) != 0 || (*(volatile const int*)&sc->steady) != 0 ||
           (*(volatile const int*)&sc->done) != 0;
}

// End of a time step (problems 2-4): the last CTA of the step's final launch to finish
// counts the step and applies the step budget.  Every CTA of that launch has finished its
// work by then, so no CTA sees the budget change in the middle of a step.
__device__ __forceinline__ void end_of_step(Scalars* sc, int nctas) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const int prev = atomicAdd(&sc->ctas_done, 1);
        if (prev == nctas - 1) {
            __threadfence();
            sc->ctas_done = 0;
            if (!halted(sc)) {
                const int n = sc->step_count + 1;
                sc->step_count = n;
                if (sc->step_limit > 0 && n >= sc->step_limit) sc->done = 1;
            }
        }
    }
}

// cal_W / cal_dW (kernel_functions_mod.f90:26-146); nrm = kernel_norm(kt, h), ih = 1/h.
// R = double: the parity arithmetic; R = float: the mixed-precision pair phase.
template <class R>
__device__ __forceinline__ R dev_W(int kt, R r, R ih, R nrm) {
    const R q = r * ih;
    R W = R(0);
    if (kt == 3) {
        if (R(0.0) <= q && q <= R(2.0)) {
            const R t = R(1.0) - R(0.5) * q, t2 = t * t, t4 = t2 * t2;
            W = t4 * (R(1.0) + R(2.0) * q);
        }
    } else if (kt == 1) {
        const R a = R(2.0) - q, b = R(1.0) - q, a3 = (a * a) * a, b3 = (b * b) * b;
        if (R(0.0) <= q && q <= R(1.0)) W = a3 - R(4.0) * b3;
        else if (R(1.0) < q && q <= R(2.0)) W = a3;
    } else if (kt == 2) {
        const R a = R(3.0) - q, b = R(2.0) - q, c = R(1.0) - q;
        const R a2 = a * a, b2 = b * b, c2 = c * c;
        const R a5 = (a2 * a2) * a, b5 = (b2 * b2) * b, c5 = (c2 * c2) * c;
        if (R(0.0) <= q && q <= R(1.0)) W = (a5 - R(6.0) * b5) + R(15.0) * c5;
        else if (R(1.0) < q && q <= R(2.0)) W = a5 - R(6.0) * b5;
        else if (R(2.0) < q && q <= R(3.0)) W = a5;
    } else if (kt == 4) {
        if (R(0.0) <= q && q <= R(2.0)) {
            const R t = R(1.0) - R(0.5) * q, t2 = t * t, t4 = t2 * t2, t6 = t4 * t2;
            W = t6 * ((R(1.0) + R(3.0) * q) + (R(35.0) * (q * q)) / R(12.0));
        }
    } else {
        if (R(0.0) <= q && q <= R(2.0)) {
            const R t = R(1.0) - R(0.5) * q, t2 = t * t, t4 = t2 * t2, t8 = t4 * t4;
            const R q2 = q * q, q3 = q2 * q;
            W = t8 * (((R(1.0) + R(4.0) * q) + (R(25.0) * q2) / R(4.0)) + R(4.0) * q3);
        }
    }
    return nrm * W;
}

template <class R>
__device__ __forceinline__ R dev_dW(int kt, R r, R ih, R m3h, R m5h, R nrm) {
    const R q = r * ih;
    R dW = R(0);
    if (kt == 3) {
        if (R(0.0) <= q && q <= R(2.0)) {
            const R t = R(1.0) - R(0.5) * q, t2 = t * t, t3 = t2 * t, t4 = t2 * t2;
            dW = -(R(2.0) * t3) * (R(1.0) + R(2.0) * q) + R(2.0) * t4;
        }
        return (nrm * dW) * ih;
    } else if (kt == 1) {
        const R a = R(2.0) - q, b = R(1.0) - q;
        if (R(0.0) <= q && q <= R(1.0)) dW = a * a - R(4.0) * (b * b);
        else if (R(1.0) < q && q <= R(2.0)) dW = a * a;
        return (nrm * dW) * m3h;
    } else if (kt == 2) {
        const R a = R(3.0) - q, b = R(2.0) - q, c = R(1.0) - q;
        const R a2 = a * a, b2 = b * b, c2 = c * c;
        const R a4 = a2 * a2, b4 = b2 * b2, c4 = c2 * c2;
        if (R(0.0) <= q && q <= R(1.0)) dW = (a4 - R(6.0) * b4) + R(15.0) * c4;
        else if (R(1.0) < q && q <= R(2.0)) dW = a4 - R(6.0) * b4;
        else if (R(2.0) < q && q <= R(3.0)) dW = a4;
        return (nrm * dW) * m5h;
    } else if (kt == 4) {
        if (R(0.0) <= q && q <= R(2.0)) {
            const R t = R(1.0) - R(0.5) * q, t2 = t * t, t4 = t2 * t2, t5 = t4 * t, t6 = t4 * t2;
            dW = -(R(3.0) * t5) * ((R(1.0) + R(3.0) * q) + (R(35.0) * (q * q)) / R(12.0)) + t6 * (R(3.0) + (R(35.0) * q) / R(6.0));
        }
        return (nrm * dW) * ih;
    } else {
        if (R(0.0) <= q && q <= R(2.0)) {
            const R t = R(1.0) - R(0.5) * q, t2 = t * t, t4 = t2 * t2, t6 = t4 * t2, t7 = t6 * t, t8 = t4 * t4;
            const R q2 = q * q, q3 = q2 * q;
            dW = -(R(4.0) * t7) * (((R(1.0) + R(4.0) * q) + (R(25.0) * q2) / R(4.0)) + R(4.0) * q3) +
                 t8 * ((R(4.0) + (R(25.0) * q) / R(2.0)) + R(12.0) * q2);
        }
        return (nrm * dW) * ih;
    }
}

// Index of (row j, col i), j <= i, in a column-packed upper triangle.
__host__ __device__ constexpr int UT(int j, int i) { return i * (i + 1) / 2 + j; }

// Gaussian elimination with partial pivoting + substitutions, the DGESV restatement of
// the oracle (first max |a| pivot, reciprocal column scaling, right-looking update).
// lu_factor overwrites A[row][col] by its LU factors and applies the row interchanges to
// the NB right-hand sides in B[c][row]; lu_subst then solves one column in place.
// Returns false on a zero pivot.  Row interchanges are rare for LS moment matrices, so
// the swap code runs only when the pivot row differs from the diagonal one.
template <int Q, int NB>
__device__ __forceinline__ bool lu_factor(double (&A)[Q][Q], double (&B)[NB][Q], double (&rpiv)[Q]) {
    bool ok = true;
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        int p = k;
        double amax = fabs(A[k][k]);
#pragma unroll
        for (int i = k + 1; i < Q; ++i) {
            const double a = fabs(A[i][k]);
            if (a > amax) { amax = a; p = i; }
        }
        if (p != k) {   // selects, not indexing by p: A and B stay in registers
#pragma unroll
            for (int r = k + 1; r < Q; ++r) {
                const bool sw = (p == r);
#pragma unroll
                for (int c = 0; c < Q; ++c) {
                    const double t0 = A[k][c], t1 = A[r][c];
                    A[k][c] = sw ? t1 : t0;
                    A[r][c] = sw ? t0 : t1;
                }
#pragma unroll
                for (int m = 0; m < NB; ++m) {
                    const double t0 = B[m][k], t1 = B[m][r];
                    B[m][k] = sw ? t1 : t0;
                    B[m][r] = sw ? t0 : t1;
                }
            }
        }
        const double piv = A[k][k];
        if (piv != 0.0) {
            const double rp = 1.0 / piv;
#pragma unroll
            for (int i = k + 1; i < Q; ++i) A[i][k] = A[i][k] * rp;
        } else {
            ok = false;
        }
        rpiv[k] = 1.0 / piv;
#pragma unroll
        for (int j = k + 1; j < Q; ++j)
#pragma unroll
            for (int i = k + 1; i < Q; ++i) A[i][j] = fma(-A[i][k], A[k][j], A[i][j]);
    }
    return ok;
}

template <int Q>
__device__ __forceinline__ void lu_subst(const double (&A)[Q][Q], const double (&rpiv)[Q], double (&b)[Q]) {
#pragma unroll
    for (int k = 0; k < Q; ++k)
#pragma unroll
        for (int i = k + 1; i < Q; ++i) b[i] = fma(-b[k], A[i][k], b[i]);
#pragma unroll
    for (int k = Q - 1; k >= 0; --k) {
        b[k] = b[k] * rpiv[k];
#pragma unroll
        for (int i = 0; i < k; ++i) b[i] = fma(-b[k], A[i][k], b[i]);
    }
}

// LU with the row interchanges recorded (pv[k] = pivot row of step k) instead of applied
// to right-hand sides; the mixed-precision solve reuses the factors for its refinement.
template <int Q>
__device__ __forceinline__ bool lu_factor_p(double (&A)[Q][Q], double (&rpiv)[Q], int (&pv)[Q]) {
    bool ok = true;
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        int p = k;
        double amax = fabs(A[k][k]);
#pragma unroll
        for (int i = k + 1; i < Q; ++i) {
            const double a = fabs(A[i][k]);
            if (a > amax) { amax = a; p = i; }
        }
        pv[k] = p;
        if (p != k) {
#pragma unroll
            for (int r = k + 1; r < Q; ++r) {
                const bool sw = (p == r);
#pragma unroll
                for (int c = 0; c < Q; ++c) {
                    const double t0 = A[k][c], t1 = A[r][c];
                    A[k][c] = sw ? t1 : t0;
                    A[r][c] = sw ? t0 : t1;
                }
            }
        }
        const double piv = A[k][k];
        if (piv != 0.0) {
            const double rp = 1.0 / piv;
#pragma unroll
            for (int i = k + 1; i < Q; ++i) A[i][k] = A[i][k] * rp;
        } else {
            ok = false;
        }
        rpiv[k] = 1.0 / piv;
#pragma unroll
        for (int j = k + 1; j < Q; ++j)
#pragma unroll
            for (int i = k + 1; i < Q; ++i) A[i][j] = fma(-A[i][k], A[k][j], A[i][j]);
    }
    return ok;
}

template <int Q>
__device__ __forceinline__ void lu_permute(const int (&pv)[Q], double (&b)[Q]) {
#pragma unroll
    for (int k = 0; k < Q; ++k) {
#pragma unroll
        for (int r = k + 1; r < Q; ++r) {
            const bool sw = (pv[k] == r);
            const double t0 = b[k], t1 = b[r];
            b[k] = sw ? t1 : t0;
            b[r] = sw ? t0 : t1;
        }
    }
}

// Mixed-precision LS solve of one right-hand side: FP64 LU of the moment matrix (whose
// sums were formed in FP32), then one step of iterative refinement against the same
// FP64 matrix: x = x0 + LU \ (b - M x0).  M is read back from the packed upper triangle.
template <int Q>
__device__ __forceinline__ void lu_solve_refined(const double (&LU)[Q][Q], const double (&rpiv)[Q],
                                                 const int (&pv)[Q], const double (&Mu)[Q * (Q + 1) / 2],
                                                 double (&b)[Q]) {
    double x[Q], r[Q];
#pragma unroll
    for (int k = 0; k < Q; ++k) x[k] = b[k];
    lu_permute<Q>(pv, x);
    lu_subst<Q>(LU, rpiv, x);
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        double s = b[i];
#pragma unroll
        for (int j = 0; j < Q; ++j) s = fma(-(i <= j ? Mu[UT(i, j)] : Mu[UT(j, i)]), x[j], s);
        r[i] = s;
    }
    lu_permute<Q>(pv, r);
    lu_subst<Q>(LU, rpiv, r);
#pragma unroll
    for (int k = 0; k < Q; ++k) b[k] = x[k] + r[k];
}

template <int Q, int NB>
__device__ __forceinline__ bool lu_solve(double (&A)[Q][Q], double (&B)[NB][Q]) {
    double rpiv[Q];
    const bool ok = lu_factor<Q, NB>(A, B, rpiv);
#pragma unroll
    for (int m = 0; m < NB; ++m) lu_subst<Q>(A, rpiv, B[m]);
    return ok;
}

// Butterfly sum over aligned groups of G lanes; every lane of the group ends with the
// same bits (IEEE addition is commutative).
template <int G>
__device__ __forceinline__ double group_sum(double v) {
#pragma unroll
    for (int off = G / 2; off >= 1; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    return v;
}
template <int G>
__device__ __forceinline__ int group_sum_i(int v) {
#pragma unroll
    for (int off = G / 2; off >= 1; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    return v;
}

// Visit the candidates of cell `key` (3x3 cells in reference order; within a cell the
// interior particles in list order, then the cell's ghosts).  Used by the parity-only
// neighbour listing, which sorts its output.
template <bool FLUID_ONLY, class F>
__device__ __forceinline__ void for_candidates(const Phys& P, const Lst& L, const int* gstart, const int* glist,
                                               int key, F&& f) {
    // f(j, sx, sy): sx, sy = position shift of j's cell (-+Lx across a periodic boundary)
    const int cx = key % P.nx, cy = key / P.nx;
    for (int dy = -1; dy <= 1; ++dy) {
        int yy = cy + dy;
        double sy = 0.0;
        if (P.periodic) {
            if (yy < 0) { yy += P.ny; sy = -P.Lx; }
            else if (yy >= P.ny) { yy -= P.ny; sy = P.Lx; }
        }
        if (yy < 0 || yy >= P.ny) continue;
        for (int dx = -1; dx <= 1; ++dx) {
            int xx = cx + dx;
            double sx = 0.0;
            if (P.periodic) {
                if (xx < 0) { xx += P.nx; sx = -P.Lx; }
                else if (xx >= P.nx) { xx -= P.nx; sx = P.Lx; }
            }
            if (xx < 0 || xx >= P.nx) continue;
            const int c = xx + yy * P.nx;
            const int ng = gstart[c + 1] - gstart[c];
            const int nf = min(L.cnt[c], P.cap - ng);
            for (int t = 0; t < nf; ++t) f(L.slots[(size_t)c * P.cap + t], sx, sy);
            if (!FLUID_ONLY)
                for (int t = 0; t < ng; ++t) f(glist[gstart[c] + t], sx, sy);
        }
    }
}

// Cell key of an interior particle, update_cell_mod.f90:53-55 (multiplication form).
__device__ __forceinline__ int cell_key_mul(const Phys& P, double x, double y, Scalars* sc) {
    double cxd = ceil(x * P.inv_h_eff), cyd = ceil(y * P.inv_h_eff);
    if (P.periodic) {   // wrapped positions lie in (0, Lx]: clamp the rounding at the ends
        if (x > 0.0 && x <= P.Lx) cxd = fmin(fmax(cxd, 1.0), (double)P.nx);
        if (y > 0.0 && y <= P.Lx) cyd = fmin(fmax(cyd, 1.0), (double)P.ny);
    }
    if (!(cxd >= 1.0 && cxd <= (double)P.nx && cyd >= 1.0 && cyd <= (double)P.ny)) {
        atomicOr(&sc->err, ERR_OUT_OF_DOMAIN);
        return -1;
    }
    return ((int)cxd - 1) + ((int)cyd - 1) * P.nx;
}

__device__ __forceinline__ void scatter_to_cell(const Phys& P, const Lst& Ln, const int* gstart, int key,
                                                int i, Scalars* sc) {
    if (key < 0) return;
    const int pos = atomicAdd(Ln.cnt + key, 1);
    const int lim = P.cap - (gstart[key + 1] - gstart[key]);
    if (pos < lim) Ln.slots[(size_t)key * P.cap + pos] = i;
    else atomicOr(&sc->err, ERR_CELL_OVERFLOW);
}

__device__ __forceinline__ void warp_max_atomic(unsigned long long* dst, double v) {
    // v >= 0 (or NaN); non-negative doubles order like their uint64 bit patterns
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, off));
    if ((threadIdx.x & 31) == 0 && v > 0.0) atomicMax(dst, (unsigned long long)__double_as_longlong(v));
}

// =======================================================================================
// Tile staging in shared memory
// =======================================================================================
constexpr int TX = 2, TY = 2;               // own cells of a tile
constexpr int HX = TX + 2, HY = TY + 2;     // halo cells
constexpr int HC = HX * HY;                 // 16 halo cells
constexpr int OC = TX * TY;                 // 4 own cells
#ifndef LSSPH_PPB
#define LSSPH_PPB 32
#endif
constexpr int PPB = LSSPH_PPB;              // particles per pass: a CTA has PPB * G threads
// Register budgets of the stage and PST kernels.  Loose: the compiler's choice (about 148
// registers per thread, 3 CTAs of 128 threads per SM).  Tight: at most 128 registers, so
// that 512 threads fit per SM, for a few spilled values.  Both compute identical results;
// which is faster depends on how many tiles a launch has, and each handle times both.
// Level 2 (FP64 single solves only): at most 102 registers, 640 threads per SM, so that a
// launch of up to 5 CTAs per SM fits one wave.
// Levels 3 and 4 (768 and 1024 threads per SM: at most 85 and 64 registers) serve the
// mixed-precision pair kernel of the split shape, which holds no FP64 solve.
__host__ __device__ constexpr int tile_min_blocks(int G, int tight) {
    return tight == 4 ? (PPB * G <= 1024 ? 1024 / (PPB * G) : 1)
         : tight == 3 ? (PPB * G <= 768 ? 768 / (PPB * G) : 1)
         : tight == 2 ? (PPB * G <= 640 ? 640 / (PPB * G) : 1)
                      : ((tight && PPB * G <= 512) ? 512 / (PPB * G) : 1);
}
static_assert(HC <= 32 && OC <= 32, "tile scans run in one warp");

struct TileHdr {
    int cnt[HC];        // staged particles per halo cell (interior + ghosts)
    int nf[HC];         // interior prefix of each halo cell
    int off[HC + 1];    // smem offset of each halo cell
    int own_off[OC + 1];
    int cell[HC];       // global cell of each halo cell (-1 outside the grid)
    int g0[HC];         // start of its ghost list
    double sx[HC], sy[HC];   // position shift of each halo cell (-+Lx across a periodic boundary)
};

// Halo cell holding staged position k (cells in staging order; empty cells skipped).
__device__ __forceinline__ int halo_cell_of(const TileHdr& T, int k) {
    int h = 0;
#pragma unroll
    for (int q = 1; q < HC; ++q) h += (k >= T.off[q]) ? 1 : 0;
    return h;
}

// Dynamic shared memory: SoA fields of up to HC*cap staged particles, their global
// indices, and the own-particle list.
struct SmemView {
    double* sums;   // [PPB][row stride]
    double *x, *y, *u, *v, *rho, *pre, *vol, *tem;
    int *idx, *own_k, *own_hc;
    unsigned short* nbr;   // in-radius lists (staged indices), entry e of thread t at nbr[e * blockDim.x + t]
};

// Per-thread in-radius list length: a lane tests at most ceil(9 cap / G) candidates.
__host__ __device__ inline int nbr_list_len(int cap, int G) { return (9 * cap + G - 1) / G; }

// Reduced sums handed from the pair phase to the solve phase, one row per particle of a
// pass: 15 moment entries + 5 x NB b entries + (PST) shift (2) + count.  The row stride is
// odd so that a warp reading one row per thread spreads over all shared-memory banks.
__host__ __device__ constexpr int sums_stride(int n) { return n | 1; }
constexpr int SUMS_MAX = sums_stride(15 + 5 * 5 + 1);

// Dynamic shared memory of one tile CTA; temperature is staged only when `tem` is set.
__host__ __device__ inline size_t tile_smem_bytes(int cap, int G, bool tem) {
    const size_t maxp = (size_t)HC * cap, maxo = (size_t)OC * cap;
    // 16-bit hit lists; the same area is the staging scratch of maxp ints
    const size_t lists = (size_t)PPB * G * nbr_list_len(cap, G) * sizeof(unsigned short);
    const size_t area = lists > maxp * sizeof(int) ? lists : maxp * sizeof(int);
    return (size_t)PPB * SUMS_MAX * sizeof(double) + maxp * ((tem ? 8 : 7) * sizeof(double) + sizeof(int)) +
           2 * maxo * sizeof(int) + ((area + 7) & ~(size_t)7);
}

// Dynamic shared memory of the FP64 split shape's pair kernel: no sums rows.
__host__ __device__ inline size_t tile_smem_bytes_fpp(int cap, int G, bool tem) {
    return tile_smem_bytes(cap, G, tem) - (size_t)PPB * SUMS_MAX * sizeof(double);
}

// with_sums = false: the layout without the sums rows (the split shape's pair kernel).
template <bool TEM>
__device__ __forceinline__ SmemView smem_view(void* raw, int cap, bool with_sums = true) {
    SmemView S;
    const int maxp = HC * cap, maxo = OC * cap;
    double* d = static_cast<double*>(raw);
    S.sums = with_sums ? d : nullptr;
    if (with_sums) d += PPB * SUMS_MAX;
    S.x = d; S.y = d + maxp; S.u = d + 2 * maxp; S.v = d + 3 * maxp; S.rho = d + 4 * maxp;
    S.pre = d + 5 * maxp; S.vol = d + 6 * maxp; S.tem = TEM ? d + 7 * maxp : nullptr;
    int* q = reinterpret_cast<int*>(d + (TEM ? 8 : 7) * maxp);
    S.idx = q; S.own_k = q + maxp; S.own_hc = q + maxp + maxo;
    S.nbr = reinterpret_cast<unsigned short*>(q + maxp + 2 * maxo);
    return S;
}

__device__ __forceinline__ int warp_incl_scan(int v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, v, off);
        if (lane >= off) v += t;
    }
    return v;
}

// Stage the lists of the tile whose halo cell (0,0) is global cell (cx0, cy0): counts,
// reference-order index lists (interior particles ascending, then the ghost list) and the
// own-particle list.  Own particles are the interior particles of the TX x TY own cells.
// All global loads of a phase are independent of each other.  Ends with a barrier.
template <bool FLUID_ONLY, class View>
__device__ __forceinline__ void stage_lists(const Phys& P, const Lst& L, const int* __restrict__ gstart,
                                            const int* __restrict__ glist, int cx0, int cy0, TileHdr& T,
                                            const View& S) {
    const int tid = threadIdx.x;
    int c = -1, g0 = 0;
    if (tid < HC) {
        int cx = cx0 + tid % HX, cy = cy0 + tid / HX;
        double sx = 0.0, sy = 0.0;
        if (P.periodic) {   // halo cells past an edge wrap; the even cell count keeps own cells inside
            if (cx < 0) { cx += P.nx; sx = -P.Lx; }
            else if (cx >= P.nx) { cx -= P.nx; sx = P.Lx; }
            if (cy < 0) { cy += P.ny; sy = -P.Lx; }
            else if (cy >= P.ny) { cy -= P.ny; sy = P.Lx; }
        }
        T.sx[tid] = sx;
        T.sy[tid] = sy;
        int nf = 0, ng = 0;
        if (cx >= 0 && cx < P.nx && cy >= 0 && cy < P.ny) {
            c = cx + cy * P.nx;
            g0 = __ldg(gstart + c);
            // a cell never stages more than cap particles, whatever its counters say (a
            // counter past cap has already raised the cell-overflow error)
            const int gc = min(__ldg(gstart + c + 1) - g0, P.cap);
            nf = max(0, min(__ldg(L.cnt + c), P.cap - gc));
            ng = FLUID_ONLY ? 0 : gc;
        }
        T.nf[tid] = nf;
        T.cnt[tid] = nf + ng;
        T.cell[tid] = c;
        T.g0[tid] = g0;
    }
    __syncthreads();
    if (tid < 32) {
        const int v = tid < HC ? T.cnt[tid] : 0;
        const int incl = warp_incl_scan(v);
        if (tid < HC) T.off[tid + 1] = incl;
        if (tid == 0) T.off[0] = 0;
        int w = 0;
        if (tid < OC) w = T.nf[(1 + tid % TX) + (1 + tid / TX) * HX];
        const int inclw = warp_incl_scan(w);
        if (tid < OC) T.own_off[tid + 1] = inclw;
        if (tid == 0) T.own_off[0] = 0;
    }
    __syncthreads();
    // every staged index is one independent load, spread over all threads; interior
    // indices go to a scratch list (the hit-list area, idle while staging) to be ranked
    const int n = T.off[HC];
    int* tmp = reinterpret_cast<int*>(S.nbr);
    for (int k = tid; k < n; k += blockDim.x) {
        const int h = halo_cell_of(T, k);
        const int sl = k - T.off[h], nfh = T.nf[h], ch = T.cell[h];
        if (sl < nfh) tmp[k] = __ldg(L.slots + (size_t)ch * P.cap + sl);
        else S.idx[k] = __ldg(glist + T.g0[h] + (sl - nfh));
    }
    __syncthreads();
    // each cell's interior indices in ascending order (the reference's list order): every
    // index counts the smaller ones of its cell and goes to that rank
    for (int k = tid; k < n; k += blockDim.x) {
        const int h = halo_cell_of(T, k);
        const int base = T.off[h], sl = k - base, nfh = T.nf[h];
        if (sl < nfh) {
            const int v = tmp[k];
            int r = 0;
            for (int q = 0; q < nfh; ++q) r += (tmp[base + q] < v) ? 1 : 0;
            S.idx[base + r] = v;
            const int hx = h % HX, hy = h / HX;
            if (hx >= 1 && hx <= TX && hy >= 1 && hy <= TY) {
                const int ob = T.own_off[(hx - 1) + (hy - 1) * TX];
                S.own_k[ob + sl] = k;
                S.own_hc[ob + sl] = h;
            }
        }
    }
    __syncthreads();
}

// Lists, then the SoA FP64 fields of every staged particle.
template <bool FLUID_ONLY, bool WITH_TEM>
__device__ __forceinline__ void stage_halo(const Phys& P, const Fld& F, const Lst& L, const int* __restrict__ gstart,
                                           const int* __restrict__ glist, int cx0, int cy0, TileHdr& T,
                                           const SmemView& S) {
    stage_lists<FLUID_ONLY>(P, L, gstart, glist, cx0, cy0, T, S);
    const int n = T.off[HC];
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const int j = S.idx[k];
        double xj = __ldg(F.x + j), yj = __ldg(F.y + j);
        if (P.periodic) {   // x_j + shift, so that staged x_j - x_i is the periodic offset
            const int h = halo_cell_of(T, k);
            xj = xj + T.sx[h];
            yj = yj + T.sy[h];
        }
        S.x[k] = xj;
        S.y[k] = yj;
        S.u[k] = __ldg(F.u + j);
        S.v[k] = __ldg(F.v + j);
        S.rho[k] = __ldg(F.rho + j);
        S.pre[k] = __ldg(F.pre + j);
        S.vol[k] = __ldg(F.vol + j);
        if (WITH_TEM) S.tem[k] = __ldg(F.tem + j);
    }
    __syncthreads();
}

// ---- mixed-precision staging -------------------------------------------------------------
// Positions as FP32 offsets from the FP64 origin of the tile's halo corner cell (at most
// 4 cell widths, so an offset carries ~2e-7 h_eff of rounding); fields as FP32 offsets
// from FP64 reference values (those of the first staged particle); volumes in FP32.
// Pair offsets x_j - x_i are then plain FP32 differences.  Hit lists are 16-bit.
struct SmemMx {
    double* sums;                                       // [PPB][row stride], as in SmemView
    float *ox, *oy, *u, *v, *rho, *pre, *vol, *tem;
    int *idx, *own_k, *own_hc;
    unsigned short* nbr;
};

__host__ __device__ inline size_t tile_smem_bytes_mx(int cap, int G, bool tem) {
    const size_t maxp = (size_t)HC * cap, maxo = (size_t)OC * cap;
    const size_t lists = (size_t)PPB * G * nbr_list_len(cap, G);
    return (size_t)PPB * SUMS_MAX * sizeof(double) + maxp * ((tem ? 8 : 7) * sizeof(float) + sizeof(int)) +
           2 * maxo * sizeof(int) + lists * sizeof(unsigned short);
}

// The staged arrays of a mixed tile from f on; sums: the reduced-sums rows (or NULL).
template <bool TEM>
__device__ __forceinline__ SmemMx smem_view_mx_at(double* sums, float* f, int cap) {
    SmemMx S;
    const int maxp = HC * cap, maxo = OC * cap;
    S.sums = sums;
    S.ox = f; S.oy = f + maxp; S.u = f + 2 * maxp; S.v = f + 3 * maxp; S.rho = f + 4 * maxp;
    S.pre = f + 5 * maxp; S.vol = f + 6 * maxp; S.tem = TEM ? f + 7 * maxp : nullptr;
    int* q = reinterpret_cast<int*>(f + (TEM ? 8 : 7) * maxp);
    S.idx = q; S.own_k = q + maxp; S.own_hc = q + maxp + maxo;
    S.nbr = reinterpret_cast<unsigned short*>(q + maxp + 2 * maxo);
    return S;
}

template <bool TEM>
__device__ __forceinline__ SmemMx smem_view_mx(void* raw, int cap) {
    double* d = static_cast<double*>(raw);
    return smem_view_mx_at<TEM>(d, reinterpret_cast<float*>(d + PPB * SUMS_MAX), cap);
}

// Shared memory of a pair CTA of the split shape: the mixed tile without the sums rows.
__host__ __device__ inline size_t tile_smem_bytes_mxp(int cap, int G, bool tem) {
    return tile_smem_bytes_mx(cap, G, tem) - (size_t)PPB * SUMS_MAX * sizeof(double);
}

// Field reference values of a staged tile (FP64); offsets are taken against them.
struct TileRef {
    double u, v, rho, pre, tem;
};

template <bool WITH_TEM>
__device__ __forceinline__ TileRef stage_fields_mx(const Phys& P, const Fld& F, int cx0, int cy0, const TileHdr& T,
                                                   const SmemMx& S) {
    TileRef R{0.0, 0.0, 0.0, 0.0, 0.0};
    const int n = T.off[HC];
    if (n > 0) {
        const int j0 = S.idx[0];
        R.u = __ldg(F.u + j0); R.v = __ldg(F.v + j0); R.rho = __ldg(F.rho + j0); R.pre = __ldg(F.pre + j0);
        if (WITH_TEM) R.tem = __ldg(F.tem + j0);
    }
    // positions from the split-precision copy in HBM: a particle of halo cell (hx, hy) sits at
    // (hx, hy) * cw + (ox, oy) from the tile's halo corner, which also holds for a wrapped
    // periodic neighbour (its cell origin moved by -+Lx = -+nx cw).  The cell offset is added
    // in FP64 and the sum rounded once: an FP32 cell width would shift every particle of a
    // halo column by the same rounding error, a bias between the columns' pair offsets.
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const int j = S.idx[k];
        const int h = halo_cell_of(T, k);
        S.ox[k] = (float)((double)__ldg(F.ox + j) + (double)(h % HX) * P.cw);
        S.oy[k] = (float)((double)__ldg(F.oy + j) + (double)(h / HX) * P.cw);
        S.u[k] = (float)(__ldg(F.u + j) - R.u);
        S.v[k] = (float)(__ldg(F.v + j) - R.v);
        S.rho[k] = (float)(__ldg(F.rho + j) - R.rho);
        S.pre[k] = (float)(__ldg(F.pre + j) - R.pre);
        S.vol[k] = (float)__ldg(F.vol + j);
        if (WITH_TEM) S.tem[k] = (float)(__ldg(F.tem + j) - R.tem);
    }
    __syncthreads();
    return R;
}


// Visit the staged candidates of an own particle in halo cell hc: 3x3 cells in reference
// order; lane `lane` of a G-lane group takes every G-th candidate of the concatenation.
// The three cells of a halo row are staged next to each other, so each row is one
// contiguous range of staged positions (in the reference's dx order).
template <int G, class Fn>
__device__ __forceinline__ void for_tile_candidates(const TileHdr& T, int hc, int lane, Fn&& f) {
    int base = 0;
#pragma unroll 1
    for (int dy = -1; dy <= 1; ++dy) {
        const int lo = T.off[hc - 1 + dy * HX], hi = T.off[hc + 2 + dy * HX];
        int k = lo + ((G == 1) ? 0 : ((lane - base) & (G - 1)));
#pragma unroll 4
        for (; k < hi; k += G) f(k);
        base += hi - lo;
    }
}

// Mixed-precision two-phase neighbour loop (see tile_pairs): FP32 cutoff test on the
// staged offsets, 16-bit hits, f(k, x_j - x_i, y_j - y_i) over the hits.  At the cutoff
// W and its gradient are zero, so a pair that the FP32 test classifies differently from
// FP64 contributes nothing either way.
template <int G, class Fn>
__device__ __forceinline__ int tile_pairs_mx(const TileHdr& T, const SmemMx& S, bool active, int hc, int lane,
                                             int skip, float oxi, float oyi, float heff2, Fn&& f) {
    int nl = 0;
    const int stride = blockDim.x;
    unsigned short* list = S.nbr + threadIdx.x;
    if (active) {
        for_tile_candidates<G>(T, hc, lane, [&](int k) {
            const float xji = S.ox[k] - oxi;
            const float yji = S.oy[k] - oyi;
            if (k != skip && !(xji * xji + yji * yji > heff2)) {
                list[nl * stride] = (unsigned short)k;
                ++nl;
            }
        });
    }
    auto body = [&](int k) { f(k, S.ox[k] - oxi, S.oy[k] - oyi); };
    if constexpr (G == 1) {
#pragma unroll 2
        for (int t = 0; t < nl; ++t) body(list[t * stride]);
        return nl;
    } else {
        int incl = nl;
#pragma unroll
        for (int off = 1; off < G; off <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, off, G);
            if (lane >= off) incl += v;
        }
        const int total = __shfl_sync(0xffffffffu, incl, G - 1, G);
        int bases[G];
#pragma unroll
        for (int q = 0; q < G; ++q) bases[q] = __shfl_sync(0xffffffffu, incl - nl, q, G);
        const int lane0 = (int)threadIdx.x - lane;
#pragma unroll 2
        for (int pidx = lane; pidx < total; pidx += G) {
            int o = 0, bo = bases[0];
#pragma unroll
            for (int q = 1; q < G; ++q) {
                const bool ge = pidx >= bases[q];
                o = ge ? q : o;
                bo = ge ? bases[q] : bo;
            }
            body(S.nbr[(pidx - bo) * stride + lane0 + o]);
        }
        return total;
    }
}

// Two-phase neighbour loop.  Phase A: the cutoff test r^2 <= h_eff^2 over this lane's
// candidates (same arithmetic as the reference, LSSPH_A_mod.f90:121-124), appending the
// hits in visiting order to this thread's list.  Phase B: the pair body over the hits
// only, so a warp no longer runs the full pair body for candidates most lanes reject.
// With G > 1 the G lanes of a particle split its combined hit list round-robin, so every
// lane gets ceil(hits / G) pairs.  Every lane of the warp must call this (shuffles);
// inactive lanes pass active = false.  skip = own staged position (me == you), or -1.
template <int G, class Fn>
__device__ __forceinline__ int tile_pairs(const TileHdr& T, const SmemView& S, bool active, int hc, int lane,
                                          int skip, double mx, double my, double h_eff_sq, Fn&& f) {
    int nl = 0;
    const int stride = blockDim.x;
    unsigned short* list = S.nbr + threadIdx.x;
    if (active) {
        for_tile_candidates<G>(T, hc, lane, [&](int k) {
            const double xji = S.x[k] - mx;
            const double yji = S.y[k] - my;
            if (k != skip && !(xji * xji + yji * yji > h_eff_sq)) { list[nl * stride] = (unsigned short)k; ++nl; }
        });
    }
    if constexpr (G == 1) {
#pragma unroll 2
        for (int t = 0; t < nl; ++t) f(list[t * stride]);   // two pair bodies in flight
        return nl;
    } else {
        int incl = nl;
#pragma unroll
        for (int off = 1; off < G; off <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, off, G);
            if (lane >= off) incl += v;
        }
        const int total = __shfl_sync(0xffffffffu, incl, G - 1, G);
        int bases[G];
#pragma unroll
        for (int q = 0; q < G; ++q) bases[q] = __shfl_sync(0xffffffffu, incl - nl, q, G);
        const int lane0 = (int)threadIdx.x - lane;
#pragma unroll 2
        for (int pidx = lane; pidx < total; pidx += G) {
            int o = 0, bo = bases[0];
#pragma unroll
            for (int q = 1; q < G; ++q) {   // owner lane of hit pidx (selects keep bases in registers)
                const bool ge = pidx >= bases[q];
                o = ge ? q : o;
                bo = ge ? bases[q] : bo;
            }
            f(S.nbr[(pidx - bo) * stride + lane0 + o]);
        }
        return total;
    }
}

// Accumulate the LS type-A moment matrix (upper triangle) and b vectors of one pair
// (LSSPH_A_mod.f90:136-190), df[c] = f_j - f_i.
template <int NB, class R, int Q>
__device__ __forceinline__ void accumulate_A(R (&Mu)[Q * (Q + 1) / 2], R (&B)[NB][Q], R VW, const R (&a)[Q],
                                             const R (&df)[NB]) {
#pragma unroll
    for (int ii = 0; ii < Q; ++ii) {
        const R VWa = VW * a[ii];
#pragma unroll
        for (int c = 0; c < NB; ++c) B[c][ii] = fma(VWa, df[c], B[c][ii]);
#pragma unroll
        for (int jj = 0; jj <= ii; ++jj) Mu[UT(jj, ii)] = fma(VWa, a[jj], Mu[UT(jj, ii)]);
    }
}

template <class R>
__device__ __forceinline__ void basis_A(R ih1, R ih2A, R x, R y, R (&a)[5]) {
    a[0] = x * ih1;
    a[1] = y * ih1;
    a[2] = (R(0.5) * (x * x)) * ih2A;
    a[3] = (R(0.5) * (y * y)) * ih2A;
    a[4] = (x * y) * ih2A;
}

// First-order basis [x/h, y/h] (order k = 1, q = 2: the PST interpolation of the classical
// SPH models, shift_interpolate_mod.f90:43-54).
template <class R>
__device__ __forceinline__ void basis_A(R ih1, R, R x, R y, R (&a)[2]) {
    a[0] = x * ih1;
    a[1] = y * ih1;
}

template <int Q>
__device__ __forceinline__ void basis_A(const Phys& P, double x, double y, double (&a)[Q]) {
    basis_A<double>(P.ih1, P.ih2A, x, y, a);
}

// Constants of the pair phase in its working precision.
template <class R>
struct PairConst {
    R ih1, ih2A, wnorm, iWave, m3h, m5h;
    __device__ __forceinline__ explicit PairConst(const Phys& P)
        : ih1(R(P.ih1)), ih2A(R(P.ih2A)), wnorm(R(P.wnorm)), iWave(R(P.iWave)), m3h(R(P.m3h)), m5h(R(P.m5h)) {}
};

// Reduce G lanes' partial sums; FP32 partials are widened first, so the lanes combine
// in FP64 (each lane's FP32 sum spans at most ceil(P / G) neighbours).
template <int G, int N, class R>
__device__ __forceinline__ void group_reduce_to(const R (&v)[N], double (&out)[N]);

template <int G, int N>
__device__ __forceinline__ void group_reduce(double (&v)[N]) {
    if constexpr (G > 1) {
#pragma unroll
        for (int k = 0; k < N; ++k) v[k] = group_sum<G>(v[k]);
    }
}

template <int G, int N, class R>
__device__ __forceinline__ void group_reduce_to(const R (&v)[N], double (&out)[N]) {
#pragma unroll
    for (int k = 0; k < N; ++k) out[k] = (double)v[k];
    group_reduce<G>(out);
}

// ---- compensated FP32 sums of the mixed-precision pair phase ------------------------------
// Kahan summation (Kahan 1965; Higham, Accuracy and Stability of Numerical Algorithms,
// section 4.3): each FP32 sum s carries c, minus the low-order part the last additions
// dropped, so s - c is the sum to about FP32 eps^2 relative to the summands instead of
// n eps.  The file is compiled with -fmad=false and nvcc does not reassociate, so the
// correction terms are evaluated as written.
__device__ __forceinline__ void kahan_add(float& s, float& c, float t) {
    const float y = t - c;
    const float u = s + y;
    c = (u - s) - y;
    s = u;
}

// accumulate_A with compensated sums (moment matrix and b vectors).
template <int NB, int Q>
__device__ __forceinline__ void accumulate_A_kahan(float (&Mu)[Q * (Q + 1) / 2], float (&Mc)[Q * (Q + 1) / 2],
                                                   float (&B)[NB][Q], float (&Bc)[NB][Q], float VW,
                                                   const float (&a)[Q], const float (&df)[NB]) {
#pragma unroll
    for (int ii = 0; ii < Q; ++ii) {
        const float VWa = VW * a[ii];
#pragma unroll
        for (int c = 0; c < NB; ++c) kahan_add(B[c][ii], Bc[c][ii], VWa * df[c]);
#pragma unroll
        for (int jj = 0; jj <= ii; ++jj) kahan_add(Mu[UT(jj, ii)], Mc[UT(jj, ii)], VWa * a[jj]);
    }
}

// Widen compensated lane sums (s - c, formed in FP64) and combine the G lanes in FP64.
template <int G, int N>
__device__ __forceinline__ void group_reduce_kahan(const float (&v)[N], const float (&c)[N], double (&out)[N]) {
#pragma unroll
    for (int k = 0; k < N; ++k) out[k] = (double)v[k] - (double)c[k];
    group_reduce<G>(out);
}

// =======================================================================================
// k_stage: LS-SPH type-A RHS (q = 5, SPH_MODEL 3) + RK stage update + cell scatter.
// NB = number of b-vector columns: 1 (problem 1: u only), 4 (u,v,rho,p), 5 (+T).
// =======================================================================================
// Right-hand sides of the governing equations from the LS derivatives (LSSPH_A_mod.f90:
// 246-269); d[c][k] are the derivatives of field c (entries x, y, xx, yy, xy).
template <int NB>
__device__ __forceinline__ void rhs_ls(const Phys& P, const Work& W, int i, double my_rho, double my_tem,
                                       const double (&d)[NB][5], double& Ru, double& Rv, double& Rr, double& Rt) {
    Rv = 0.0; Rr = 0.0; Rt = 0.0;
    if constexpr (NB == 1) {
        Ru = (d[0][2] + d[0][3]) + W.src[i];
    } else {
        // d[0] = u, d[1] = v, d[2] = rho, d[3] = p (, d[4] = T); entries x, y, xx, yy, xy
        const double irho = 1.0 / my_rho;
        Rr = -(my_rho * (d[0][0] + d[1][1])) + P.delta * (d[2][2] + d[2][3]);
        Ru = -(d[3][0] * irho) + (P.vis_ref * irho) * (d[0][2] + d[0][3]);
        Rv = -(d[3][1] * irho) + (P.vis_ref * irho) * (d[1][2] + d[1][3]);
        Rr = Rr * P.izeta2;
        if constexpr (NB == 5) {
            Rv = Rv + ((P.alpha_ref * (my_tem - P.tem_ave)) * P.gravity);
            Ru = Ru * P.ixi2;
            Rv = Rv * P.ixi2;
            Rt = P.thermal_dif * (d[NB - 1][2] + d[NB - 1][3]);
        }
    }
}

// Tail of a stage, in pieces (RK2_mod.f90:87-108 / RK4_mod.f90:109-159): keep the RHS;
// the start-of-step and RK4 accumulator values; the new position and its cell key (which
// need the current velocity only, not the RHS); the new fields and the EOS; the scatter
// into the next cell list.  stage_advance runs them in that order for one particle.  The
// tile stage kernels (LS in FP64 and mixed precision, classical) with more than one warp
// move their particles on the warps that have no solve to do, so that the position loads
// and the scatter's atomics overlap the solve.
template <int NB>
__device__ __forceinline__ void keep_rhs(const Work& W, const StageCfg& S, int i, double Ru, double Rv, double Rr,
                                         double Rt) {
    if (S.write_rhs) {
        W.rhs_u[i] = Ru;
        if constexpr (NB >= 4) { W.rhs_v[i] = Rv; W.rhs_rho[i] = Rr; }
        if constexpr (NB == 5) W.rhs_tem[i] = Rt;
    }
}

// Start-of-step values (old) and RK4 accumulators (acc) of the fields; stage 1 takes the
// current values for both.
struct OldFields {
    double uo, vo, ro, to, ua, va, ra, ta;
};

template <int NB>
__device__ __forceinline__ OldFields load_old_fields(const Phys& P, const Work& W, const StageCfg& S, int i,
                                                     double my_u, double my_v, double my_rho, double my_tem) {
    constexpr bool p1 = (NB == 1);   // problem 1 updates u only
    OldFields o{my_u, my_v, my_rho, my_tem, my_u, my_v, my_rho, my_tem};
    if (S.stage != 1) {
        o.uo = W.u_old[i];
        if constexpr (!p1) { o.vo = W.v_old[i]; o.ro = W.rho_old[i]; }
        if constexpr (NB == 5) o.to = W.tem_old[i];
        if (P.rk != 2) {
            o.ua = W.u_acc[i];
            if constexpr (!p1) { o.va = W.v_acc[i]; o.ra = W.rho_acc[i]; }
            if constexpr (NB == 5) o.ta = W.tem_acc[i];
        }
    }
    return o;
}

// New position (problems 2-4), wrapped into the periodic box; returns its cell key when
// the stage rebuilds the cell list, else -1.
template <int NB>
__device__ __forceinline__ int stage_position(const Phys& P, const Fld& nxt, const Work& W, const StageCfg& S,
                                              Scalars* sc, int i, double my_x, double my_y, double my_u,
                                              double my_v) {
    double xo, yo, xn, yn;
    if (S.stage == 1) {
        xo = my_x; yo = my_y;
        W.x_old[i] = xo; W.y_old[i] = yo;
    } else {
        xo = W.x_old[i]; yo = W.y_old[i];
    }
    if (P.rk == 2) {
        const double dt = S.dt2;
        xn = xo + my_u * dt;
        yn = yo + my_v * dt;
    } else {
        double xa = my_x, ya = my_y;
        if (S.stage != 1) { xa = W.x_acc[i]; ya = W.y_acc[i]; }
        xa = xa + my_u * S.dt1;
        ya = ya + my_v * S.dt1;
        if (!S.last) {
            W.x_acc[i] = xa; W.y_acc[i] = ya;
            xn = xo + my_u * S.dt2;
            yn = yo + my_v * S.dt2;
        } else {
            xn = xa; yn = ya;
        }
    }
    if (P.periodic) { xn = wrap_pos(xn, P.Lx); yn = wrap_pos(yn, P.Lx); }
    nxt.x[i] = xn;
    nxt.y[i] = yn;
    if (!(isfinite(xn) && isfinite(yn))) atomicOr(&sc->err, ERR_NONFINITE);
    int nk = -1;
    if (S.do_scatter) {
        nk = cell_key_mul(P, xn, yn, sc);
        if (nk >= 0) {
            W.key[i] = nk;
            if (P.split_pos) put_split_pos(P, nxt, i, xn, yn, nk);
        }
    }
    return nk;
}

// Cell key of a stage: the new position's (problems 2-4), or the fixed one (problem 1).
template <int NB>
__device__ __forceinline__ int stage_key(const Phys& P, const Fld& nxt, const Work& W, const StageCfg& S,
                                         Scalars* sc, int i, double my_x, double my_y, double my_u, double my_v) {
    if constexpr (NB != 1) return stage_position<NB>(P, nxt, W, S, sc, i, my_x, my_y, my_u, my_v);
    int nk = -1;
    if (S.do_scatter) {
        nk = cell_key_mul(P, my_x, my_y, sc);
        if (nk >= 0) W.key[i] = nk;
    }
    return nk;
}

// New fields, EOS and volume; returns this particle's value for the U_max / steady-state
// max reductions.
template <int NB>
__device__ __forceinline__ double stage_fields(const Phys& P, const Fld& nxt, const Work& W, const StageCfg& S,
                                               Scalars* sc, int i, double my_v, double my_rho, double my_tem,
                                               double Ru, double Rv, double Rr, double Rt, const OldFields& o) {
    constexpr bool p1 = (NB == 1);
    if (S.stage == 1) {
        W.u_old[i] = o.uo;
        if constexpr (!p1) { W.v_old[i] = o.vo; W.rho_old[i] = o.ro; }
        if constexpr (NB == 5) W.tem_old[i] = o.to;
    }
    double un, vn = my_v, rn = my_rho, tn = my_tem;
    if (P.rk == 2) {
        const double dt = S.dt2;
        if constexpr (!p1) {
            vn = o.vo + Rv * dt;
            rn = o.ro + Rr * dt;
        }
        un = o.uo + Ru * dt;
        if constexpr (NB == 5) tn = o.to + Rt * dt;
    } else {
        const double ua = o.ua + Ru * S.dt1;
        double va = 0, ra = 0, ta = 0;
        if constexpr (!p1) {
            va = o.va + Rv * S.dt1;
            ra = o.ra + Rr * S.dt1;
        }
        if constexpr (NB == 5) ta = o.ta + Rt * S.dt1;
        if (!S.last) {
            W.u_acc[i] = ua;
            if constexpr (!p1) { W.v_acc[i] = va; W.rho_acc[i] = ra; }
            if constexpr (NB == 5) W.tem_acc[i] = ta;
            if constexpr (!p1) {
                vn = o.vo + Rv * S.dt2;
                rn = o.ro + Rr * S.dt2;
            }
            un = o.uo + Ru * S.dt2;
            if constexpr (NB == 5) tn = o.to + Rt * S.dt2;
        } else {
            un = ua;
            if constexpr (!p1) { vn = va; rn = ra; }
            if constexpr (NB == 5) tn = ta;
        }
    }
    nxt.u[i] = un;
    bool finite = isfinite(un);
    if constexpr (!p1) {
        nxt.v[i] = vn; nxt.rho[i] = rn;
        nxt.pre[i] = P.c_sq * (rn - P.rho_ref);
        nxt.vol[i] = P.SP_mass / rn;
        finite = finite && isfinite(vn) && isfinite(rn);
    }
    if constexpr (NB == 5) { nxt.tem[i] = tn; finite = finite && isfinite(tn); }
    if (!finite) atomicOr(&sc->err, ERR_NONFINITE);
    double red = 0.0;
    if (S.last && S.do_umax) red = un * un + vn * vn;
    if (S.last && S.do_steady) {
        red = fabs(W.f_prev[i] - un);
        W.f_prev[i] = un;
    }
    return red;
}

// The whole tail for one particle.
template <int NB>
__device__ __forceinline__ double stage_advance(const Phys& P, const Fld& nxt, const Lst& Ln,
                                                const int* __restrict__ gstart, const Work& W, const StageCfg& S,
                                                Scalars* sc, int i, double my_x, double my_y, double my_u,
                                                double my_v, double my_rho, double my_tem, double Ru, double Rv,
                                                double Rr, double Rt) {
    keep_rhs<NB>(W, S, i, Ru, Rv, Rr, Rt);
    if (S.mode == MODE_RHS_ONLY) return 0.0;
    const OldFields o = load_old_fields<NB>(P, W, S, i, my_u, my_v, my_rho, my_tem);
    const int nk = stage_key<NB>(P, nxt, W, S, sc, i, my_x, my_y, my_u, my_v);
    const double red = stage_fields<NB>(P, nxt, W, S, sc, i, my_v, my_rho, my_tem, Ru, Rv, Rr, Rt, o);
    if (S.do_scatter) scatter_to_cell(P, Ln, gstart, nk, i, sc);
    return red;
}

// New position, cell key and scatter of own particles first, first + step, ... (threads
// of a tile CTA that have no solve to do); get(o, i, x, y, u, v) reads own particle o's
// index and FP64 position and velocity.
template <int NB, class Get>
__device__ __forceinline__ void stage_move_own(const Phys& P, const Fld& nxt, const Lst& Ln,
                                               const int* __restrict__ gstart, const Work& W, const StageCfg& S,
                                               Scalars* sc, int n_own, int first, int step, Get&& get) {
    for (int o = first; o < n_own; o += step) {
        int i;
        double x, y, u, v;
        get(o, i, x, y, u, v);
        const int nk = stage_key<NB>(P, nxt, W, S, sc, i, x, y, u, v);
        if (S.do_scatter) scatter_to_cell(P, Ln, gstart, nk, i, sc);
    }
}

// FP64 pair phase of one own particle of a stage (LSSPH_A_mod.f90:102-197): the G lanes of
// the particle share its candidates (tile_pairs), and their sums are combined into Md (the
// packed upper triangle of the moment matrix) and Bd (one b vector per field).  Returns the
// in-radius count.  Every lane of the warp calls it (shuffles); inactive lanes pass
// active = false.  The fused stage kernel and the split shape's pair kernel share it, so
// both shapes form the same sums.
template <int NB, int G, int KT>
__device__ __forceinline__ int stage_pair_sums_kt(const Phys& P, const TileHdr& T, const SmemView& SM, bool active,
                                                  int ki, int hc, int lane, double (&Md)[15], double (&Bd)[NB][5]) {
    const int kt = KT ? KT : P.kt;
    constexpr int Q = 5;
    const double my_x = SM.x[ki], my_y = SM.y[ki], my_u = SM.u[ki];
    double my_v = 0, my_rho = 0, my_pre = 0, my_tem = 0;
    if constexpr (NB >= 4) { my_v = SM.v[ki]; my_rho = SM.rho[ki]; my_pre = SM.pre[ki]; }
    if constexpr (NB == 5) my_tem = SM.tem[ki];
    using R = double;
    const PairConst<R> C(P);
    R Mu[15];
    R B[NB][Q];
#pragma unroll
    for (int k = 0; k < 15; ++k) Mu[k] = R(0);
#pragma unroll
    for (int c = 0; c < NB; ++c)
#pragma unroll
        for (int k = 0; k < Q; ++k) B[c][k] = R(0);
    const int cnt = tile_pairs<G>(T, SM, active, hc, lane, ki, my_x, my_y, P.h_eff_sq, [&](int k) {
        const R xji = R(SM.x[k] - my_x);
        const R yji = R(SM.y[k] - my_y);
        const R r = sqrt(xji * xji + yji * yji);
        const R Wv = dev_W<R>(kt, r, C.ih1, C.wnorm);
        const R VW = R(SM.vol[k]) * Wv;
        R a[Q];
        basis_A<R>(C.ih1, C.ih2A, xji, yji, a);
        R df[NB];
        df[0] = R(SM.u[k] - my_u);
        if constexpr (NB >= 4) {
            df[1] = R(SM.v[k] - my_v);
            df[2] = R(SM.rho[k] - my_rho);
            df[3] = R(SM.pre[k] - my_pre);
        }
        if constexpr (NB == 5) df[4] = R(SM.tem[k] - my_tem);
        accumulate_A<NB, R>(Mu, B, VW, a, df);
    });
    group_reduce_to<G>(Mu, Md);
#pragma unroll
    for (int c = 0; c < NB; ++c) group_reduce_to<G>(B[c], Bd[c]);
    return cnt;
}

// The pair loop is compiled twice: for the Wendland C2 kernel (KERNEL_TYPE 3, the default),
// whose weight then needs no branch on the kernel type inside the loop, and for any type.
template <int NB, int G>
__device__ __forceinline__ int stage_pair_sums(const Phys& P, const TileHdr& T, const SmemView& SM, bool active,
                                               int ki, int hc, int lane, double (&Md)[15], double (&Bd)[NB][5]) {
    if (P.kt == 3) return stage_pair_sums_kt<NB, G, 3>(P, T, SM, active, ki, hc, lane, Md, Bd);
    return stage_pair_sums_kt<NB, G, 0>(P, T, SM, active, ki, hc, lane, Md, Bd);
}

// One tile of one solve (the CTA's work in both the single-solve and the batched kernel).
template <int NB, int G>
__device__ __forceinline__ void stage_body_fp64(const Phys& P, const Fld& cur, const Fld& nxt, const Lst& Lc, const Lst& Ln,
                                           const int* __restrict__ gstart, const int* __restrict__ glist,
                                           const Work& W, const StageCfg& S, Scalars* sc, int ntx, int tile) {
    pdl_wait();
    const bool stop = halted(sc);   // consumed after staging, so its load overlaps the staging loads
    constexpr int Q = 5;
    constexpr int SR = sums_stride(15 + 5 * NB + 1);
    static_assert(SR <= SUMS_MAX, "reduced sums overflow");
    __shared__ TileHdr T;
    extern __shared__ double smem_raw[];
    const SmemView SM = smem_view<NB == 5>(smem_raw, P.cap);
    const int tx = tile % ntx, ty = tile / ntx;
    stage_halo<false, NB == 5>(P, cur, Lc, gstart, glist, tx * TX - 1, ty * TY - 1, T, SM);
    pdl_release();
    if (stop) return;
    const int n_own = T.own_off[OC];
    const int lane = threadIdx.x & (G - 1);
    const bool early = S.mode == MODE_STAGE;
    auto own = [&](int o, int& i, double& x, double& y, double& u, double& v) {
        const int ki = SM.own_k[o];
        i = SM.idx[ki];
        x = SM.x[ki];
        y = SM.y[ki];
        u = SM.u[ki];
        v = NB >= 4 ? SM.v[ki] : 0.0;
    };
    for (int ob = 0; ob < n_own; ob += PPB) {
        // ---- pair phase: G lanes per particle ----
        {
            const int slot = (int)threadIdx.x / G;
            const int o = ob + slot;
            const bool active = o < n_own;
            int ki = 0, hc = 0;
            if (active) { ki = SM.own_k[o]; hc = SM.own_hc[o]; }
            double Md[15], Bd[NB][Q];
            const int cnt = stage_pair_sums<NB, G>(P, T, SM, active, ki, hc, lane, Md, Bd);
            if (active && lane == 0) {
                double* sm = SM.sums + slot * SR;
#pragma unroll
                for (int k = 0; k < 15; ++k) sm[k] = Md[k];
#pragma unroll
                for (int c = 0; c < NB; ++c)
#pragma unroll
                    for (int k = 0; k < Q; ++k) sm[15 + 5 * c + k] = Bd[c][k];
                sm[SR - 1] = (double)cnt;
            }
        }
        __syncthreads();
        // ---- solve phase: one thread per particle (DGESV, LSSPH_A_mod.f90:203-241) ----
        double red = 0.0;
        const int o = ob + (int)threadIdx.x;
        if ((int)threadIdx.x < PPB && o < n_own) {
            double* sm = SM.sums + threadIdx.x * SR;
            const int ki = SM.own_k[o];
            const int i = SM.idx[ki];
            const int cnt = (int)sm[SR - 1];
            double my_v = 0, my_rho = 0, my_tem = 0;
            if constexpr (NB >= 4) { my_v = SM.v[ki]; my_rho = SM.rho[ki]; }
            if constexpr (NB == 5) my_tem = SM.tem[ki];
            double d[NB][Q];
            {
                double A[Q][Q];
                double B[NB][Q];
#pragma unroll
                for (int r = 0; r < Q; ++r)
#pragma unroll
                    for (int c = 0; c < Q; ++c) A[r][c] = (r <= c) ? sm[UT(r, c)] : sm[UT(c, r)];
#pragma unroll
                for (int c = 0; c < NB; ++c)
#pragma unroll
                    for (int k = 0; k < Q; ++k) B[c][k] = sm[15 + 5 * c + k];
                if (cnt >= Q) {
                    if (!lu_solve<Q, NB>(A, B)) atomicOr(&sc->warn, WARN_SINGULAR);
#pragma unroll
                    for (int c = 0; c < NB; ++c)
#pragma unroll
                        for (int k = 0; k < Q; ++k) d[c][k] = B[c][k] * (k < 2 ? P.ih1 : P.ih2A);
                } else {
#pragma unroll
                    for (int c = 0; c < NB; ++c)
#pragma unroll
                        for (int k = 0; k < Q; ++k) d[c][k] = 0.0;
                }
            }
            double Ru, Rv, Rr, Rt;
            rhs_ls<NB>(P, W, i, my_rho, my_tem, d, Ru, Rv, Rr, Rt);
            keep_rhs<NB>(W, S, i, Ru, Rv, Rr, Rt);
            if (early) {
                const OldFields of = load_old_fields<NB>(P, W, S, i, SM.u[ki], my_v, my_rho, my_tem);
                red = stage_fields<NB>(P, nxt, W, S, sc, i, my_v, my_rho, my_tem, Ru, Rv, Rr, Rt, of);
            }
        } else if (G > 1 && early && ob == 0 && (int)threadIdx.x >= PPB) {
            // the warps idle in the solve phase move every own particle (the new position
            // needs no RHS), key it and append it to the next cell list
            stage_move_own<NB>(P, nxt, Ln, gstart, W, S, sc, n_own, (int)threadIdx.x - PPB, blockDim.x - PPB, own);
        }
        if (S.mode == MODE_STAGE && S.last && (S.do_umax || S.do_steady))
            warp_max_atomic(S.do_umax ? &sc->umax2 : &sc->dfmax, red);
        __syncthreads();
    }
    if constexpr (G == 1)
        if (early) stage_move_own<NB>(P, nxt, Ln, gstart, W, S, sc, n_own, threadIdx.x, blockDim.x, own);
}


// FP64 LS solve of one particle's sums row in place, as the fused FP64 kernels solve it
// (DGESV, LSSPH_A_mod.f90:203-241, no refinement); the solution replaces the b sums, scaled
// by the basis factors when SCALE; cnt < Q leaves zeros.
template <int Q, int NB, bool SCALE>
__device__ __forceinline__ void solve_row_plain(const Phys& P, double* row, int cnt, Scalars* sc) {
    if (cnt >= Q) {
        double A[Q][Q];
        double B[NB][Q];
#pragma unroll
        for (int r = 0; r < Q; ++r)
#pragma unroll
            for (int c = 0; c < Q; ++c) A[r][c] = (r <= c) ? row[UT(r, c)] : row[UT(c, r)];
#pragma unroll
        for (int c = 0; c < NB; ++c)
#pragma unroll
            for (int k = 0; k < Q; ++k) B[c][k] = row[15 + 5 * c + k];
        if (!lu_solve<Q, NB>(A, B)) atomicOr(&sc->warn, WARN_SINGULAR);
#pragma unroll
        for (int c = 0; c < NB; ++c)
#pragma unroll
            for (int k = 0; k < Q; ++k) row[15 + 5 * c + k] = SCALE ? B[c][k] * (k < 2 ? P.ih1 : P.ih2A) : B[c][k];
    } else {
#pragma unroll
        for (int k = 15; k < 15 + 5 * NB; ++k) row[k] = 0.0;
    }
}

// ---- mixed precision: LS solve of one particle's sums row in place ----------------------
// FP64 LU of the moment matrix (packed upper triangle at row[0..14]), then per right-hand
// side the DGESV substitutions plus one refinement step; the solution replaces the b sums
// (scaled by the basis factors when SCALE).  cnt < Q leaves zeros, as the FP64 path does.
template <int Q, int NB, bool SCALE>
__device__ __forceinline__ void solve_row_refined(const Phys& P, double* row, int cnt, Scalars* sc) {
    if (cnt >= Q) {
        double A[Q][Q];
#pragma unroll
        for (int r = 0; r < Q; ++r)
#pragma unroll
            for (int c = 0; c < Q; ++c) A[r][c] = (r <= c) ? row[UT(r, c)] : row[UT(c, r)];
        double Mr[Q * (Q + 1) / 2];   // the matrix stays in registers for every refinement
#pragma unroll
        for (int k = 0; k < Q * (Q + 1) / 2; ++k) Mr[k] = row[k];
        double rpiv[Q];
        int pv[Q];
        if (!lu_factor_p<Q>(A, rpiv, pv)) atomicOr(&sc->warn, WARN_SINGULAR);
#pragma unroll 1
        for (int c = 0; c < NB; ++c) {
            double b[Q];
#pragma unroll
            for (int k = 0; k < Q; ++k) b[k] = row[15 + 5 * c + k];
            lu_solve_refined<Q>(A, rpiv, pv, Mr, b);
#pragma unroll
            for (int k = 0; k < Q; ++k) row[15 + 5 * c + k] = SCALE ? b[k] * (k < 2 ? P.ih1 : P.ih2A) : b[k];
        }
    } else {
#pragma unroll
        for (int k = 15; k < 15 + 5 * NB; ++k) row[k] = 0.0;
    }
}

// Mixed-precision pair phase of one own particle (FP32 offsets and field references staged
// in shared memory): the stage's sums (LSSPH_A_mod.f90:102-197) or, with PST, the shift
// interpolation's sums and the shift vector sums (shift_interpolate_mod.f90:120-190), each
// lane's FP32 partial sums (compensated with COMP) combined over the particle's G lanes in
// FP64.  Returns the in-radius count.  Every lane of the warp calls it (shuffles).  The
// fused and split mixed kernels share it; KT as stage_pair_sums_kt.
template <int NB, int G, bool COMP, bool PST, int KT>
__device__ __forceinline__ int mx_pair_sums_kt(const Phys& P, const TileHdr& T, const SmemMx& SM, bool active,
                                               int ki, int hc, int lane, double (&Md)[15], double (&Bd)[NB][5],
                                               double (&sd)[2]) {
    constexpr bool TEM = PST ? (NB == 4) : (NB == 5);
    constexpr int Q = 5;
    const int kt = KT ? KT : P.kt;
    const float heff2 = (float)P.h_eff_sq;
    const PairConst<float> C(P);
    const float oxi = SM.ox[ki], oyi = SM.oy[ki];
    const float my_u = SM.u[ki];
    float my_v = 0.f, my_rho = 0.f, my_pre = 0.f, my_tem = 0.f;
    if constexpr (PST || NB >= 4) { my_v = SM.v[ki]; my_rho = SM.rho[ki]; }
    if constexpr (!PST && NB >= 4) my_pre = SM.pre[ki];
    if constexpr (TEM) my_tem = SM.tem[ki];
    float Mu[15], Mc[15];
    float B[NB][Q], Bc[NB][Q];
    float sxy[2] = {0.f, 0.f}, sxc[2] = {0.f, 0.f};
#pragma unroll
    for (int k = 0; k < 15; ++k) { Mu[k] = 0.f; Mc[k] = 0.f; }
#pragma unroll
    for (int c = 0; c < NB; ++c)
#pragma unroll
        for (int k = 0; k < Q; ++k) { B[c][k] = 0.f; Bc[c][k] = 0.f; }
    const int cnt = tile_pairs_mx<G>(T, SM, active, hc, lane, ki, oxi, oyi, heff2, [&](int k, float xji, float yji) {
        const float r = sqrtf(xji * xji + yji * yji);
        const float Wv = dev_W<float>(kt, r, C.ih1, C.wnorm);
        const float Vj = SM.vol[k];
        const float VW = Vj * Wv;
        if constexpr (PST) {
            const float dWdr = dev_dW<float>(kt, r, C.ih1, C.m3h, C.m5h, C.wnorm);
            const float rinv = 1.f / r;
            const float gx = ((dWdr * (-xji)) * rinv) * Vj;
            const float gy = ((dWdr * (-yji)) * rinv) * Vj;
            const float t = Wv * C.iWave, t2 = t * t, t4 = t2 * t2;
            const float fac = 1.f + 0.2f * t4;
            if constexpr (COMP) {
                kahan_add(sxy[0], sxc[0], fac * gx);
                kahan_add(sxy[1], sxc[1], fac * gy);
            } else {
                sxy[0] = fmaf(fac, gx, sxy[0]);
                sxy[1] = fmaf(fac, gy, sxy[1]);
            }
        }
        float a[Q];
        basis_A<float>(C.ih1, C.ih2A, xji, yji, a);
        float df[NB];
        df[0] = SM.u[k] - my_u;
        if constexpr (PST) {
            df[1] = SM.v[k] - my_v;
            df[2] = SM.rho[k] - my_rho;
            if constexpr (NB == 4) df[3] = SM.tem[k] - my_tem;
        } else {
            if constexpr (NB >= 4) {
                df[1] = SM.v[k] - my_v;
                df[2] = SM.rho[k] - my_rho;
                df[3] = SM.pre[k] - my_pre;
            }
            if constexpr (NB == 5) df[4] = SM.tem[k] - my_tem;
        }
        if constexpr (COMP) accumulate_A_kahan<NB, Q>(Mu, Mc, B, Bc, VW, a, df);
        else accumulate_A<NB, float>(Mu, B, VW, a, df);
    });
    if constexpr (COMP) {
        group_reduce_kahan<G>(Mu, Mc, Md);
#pragma unroll
        for (int c = 0; c < NB; ++c) group_reduce_kahan<G>(B[c], Bc[c], Bd[c]);
        if constexpr (PST) group_reduce_kahan<G>(sxy, sxc, sd);
    } else {
        group_reduce_to<G>(Mu, Md);
#pragma unroll
        for (int c = 0; c < NB; ++c) group_reduce_to<G>(B[c], Bd[c]);
        if constexpr (PST) group_reduce_to<G>(sxy, sd);
    }
    return cnt;
}

template <int NB, int G, bool COMP, bool PST>
__device__ __forceinline__ int mx_pair_sums(const Phys& P, const TileHdr& T, const SmemMx& SM, bool active, int ki,
                                            int hc, int lane, double (&Md)[15], double (&Bd)[NB][5],
                                            double (&sd)[2]) {
    if (P.kt == 3) return mx_pair_sums_kt<NB, G, COMP, PST, 3>(P, T, SM, active, ki, hc, lane, Md, Bd, sd);
    return mx_pair_sums_kt<NB, G, COMP, PST, 0>(P, T, SM, active, ki, hc, lane, Md, Bd, sd);
}

// Mixed-precision stage: FP32 staging and pair phase (offsets from FP64 cell origins and
// field references), lanes combined in FP64, FP64 solve (COMP: compensated lane sums and one
// refinement step of the solve), FP64 update.
template <int NB, int G, bool COMP>
__device__ __forceinline__ void stage_body_mx(const Phys& P, const Fld& cur, const Fld& nxt, const Lst& Lc,
                                              const Lst& Ln, const int* __restrict__ gstart,
                                              const int* __restrict__ glist, const Work& W, const StageCfg& S,
                                              Scalars* sc, int ntx, int tile) {
    pdl_wait();
    const bool stop = halted(sc);
    constexpr int Q = 5;
    constexpr int SR = sums_stride(15 + 5 * NB + 1);
    static_assert(SR <= SUMS_MAX, "reduced sums overflow");
    __shared__ TileHdr T;
    extern __shared__ double smem_raw[];
    const SmemMx SM = smem_view_mx<NB == 5>(smem_raw, P.cap);
    const int tx = tile % ntx, ty = tile / ntx;
    const int cx0 = tx * TX - 1, cy0 = ty * TY - 1;
    stage_lists<false>(P, Lc, gstart, glist, cx0, cy0, T, SM);
    stage_fields_mx<NB == 5>(P, cur, cx0, cy0, T, SM);
    pdl_release();
    if (stop) return;
    const int n_own = T.own_off[OC];
    const int lane = threadIdx.x & (G - 1);
    const bool early = S.mode == MODE_STAGE;
    auto own = [&](int o, int& i, double& x, double& y, double& u, double& v) {
        i = SM.idx[SM.own_k[o]];
        x = cur.x[i];
        y = cur.y[i];
        u = cur.u[i];
        v = NB >= 4 ? cur.v[i] : 0.0;
    };
    for (int ob = 0; ob < n_own; ob += PPB) {
        {
            const int slot = (int)threadIdx.x / G;
            const int o = ob + slot;
            const bool active = o < n_own;
            int ki = 0, hc = 0;
            if (active) { ki = SM.own_k[o]; hc = SM.own_hc[o]; }
            double Md[15], Bd[NB][Q], sd[2];
            const int cnt = mx_pair_sums<NB, G, COMP, false>(P, T, SM, active, ki, hc, lane, Md, Bd, sd);
            if (active && lane == 0) {
                double* sm = SM.sums + slot * SR;
#pragma unroll
                for (int k = 0; k < 15; ++k) sm[k] = Md[k];
#pragma unroll
                for (int c = 0; c < NB; ++c)
#pragma unroll
                    for (int k = 0; k < Q; ++k) sm[15 + 5 * c + k] = Bd[c][k];
                sm[SR - 1] = (double)cnt;
            }
        }
        __syncthreads();
        double red = 0.0;
        const int o = ob + (int)threadIdx.x;
        if ((int)threadIdx.x < PPB && o < n_own) {
            double* sm = SM.sums + threadIdx.x * SR;
            const int i = SM.idx[SM.own_k[o]];
            // the particle's own FP64 state (loads issued before the solve they do not need)
            const double my_u = cur.u[i];
            double my_v = 0, my_rho = 0, my_tem = 0;
            if constexpr (NB >= 4) { my_v = cur.v[i]; my_rho = cur.rho[i]; }
            if constexpr (NB == 5) my_tem = cur.tem[i];
            if constexpr (COMP) solve_row_refined<Q, NB, true>(P, sm, (int)sm[SR - 1], sc);
            else solve_row_plain<Q, NB, true>(P, sm, (int)sm[SR - 1], sc);
            double d[NB][Q];
#pragma unroll
            for (int c = 0; c < NB; ++c)
#pragma unroll
                for (int k = 0; k < Q; ++k) d[c][k] = sm[15 + 5 * c + k];
            double Ru, Rv, Rr, Rt;
            rhs_ls<NB>(P, W, i, my_rho, my_tem, d, Ru, Rv, Rr, Rt);
            keep_rhs<NB>(W, S, i, Ru, Rv, Rr, Rt);
            if (early) {
                const OldFields of = load_old_fields<NB>(P, W, S, i, my_u, my_v, my_rho, my_tem);
                red = stage_fields<NB>(P, nxt, W, S, sc, i, my_v, my_rho, my_tem, Ru, Rv, Rr, Rt, of);
            }
        } else if (G > 1 && early && ob == 0 && (int)threadIdx.x >= PPB) {
            // the warps idle in the solve phase move the own particles (FP64 state from HBM)
            stage_move_own<NB>(P, nxt, Ln, gstart, W, S, sc, n_own, (int)threadIdx.x - PPB, blockDim.x - PPB, own);
        }
        if (S.mode == MODE_STAGE && S.last && (S.do_umax || S.do_steady))
            warp_max_atomic(S.do_umax ? &sc->umax2 : &sc->dfmax, red);
        __syncthreads();
    }
    if constexpr (G == 1)
        if (early) stage_move_own<NB>(P, nxt, Ln, gstart, W, S, sc, n_own, threadIdx.x, blockDim.x, own);
}

// =======================================================================================
// Classical SPH (classical_SPH_mod.f90:26-169): SPH_MODEL 1 (sum model for the pressure
// gradient) and 2 (difference model).  Kernel-gradient sums replace the LS solve:
//   du_dx = sum gx (u_j - u_i), dv_dy = sum gy (v_j - v_i), dp = sum g (p_j +/- p_i),
//   L f   = sum 2 V_j dW/r (f_i - f_j)  for f = u, v, rho (, T),
// with x_ij = x_i - x_j, g = dW x_ij / r V_j.  Same tile staging and two-phase pair loop as
// the LS kernel; the reduced sums go to the stage update directly.
// =======================================================================================
template <int NB>
__device__ __forceinline__ void rhs_classical(const Phys& P, const Work& W, int i, double my_rho, double my_tem,
                                              const double* s, double& Ru, double& Rv, double& Rr, double& Rt) {
    // s: du_dx, dv_dy, dp_dx, dp_dy, Lu, Lv, Lrho (, LT); problem 1: Lu only
    Rv = 0.0; Rr = 0.0; Rt = 0.0;
    if constexpr (NB == 1) {
        Ru = s[0] + W.src[i];
    } else {
        Rr = -(my_rho * (s[0] + s[1])) + P.delta * s[6];
        Ru = -(s[2] / my_rho) + (P.vis_ref / my_rho) * s[4];
        Rv = -(s[3] / my_rho) + (P.vis_ref / my_rho) * s[5];
        Rr = Rr / P.zeta_sq;
        if constexpr (NB == 5) {
            Rv = Rv + ((P.alpha_ref * (my_tem - P.tem_ave)) * P.gravity);
            Ru = Ru / P.xi_sq;
            Rv = Rv / P.xi_sq;
            Rt = P.thermal_dif * s[7];
        }
    }
}

template <int NB, int G>
__device__ __forceinline__ void stage_body_classical(const Phys& P, const Fld& cur, const Fld& nxt, const Lst& Lc,
                                                     const Lst& Ln, const int* __restrict__ gstart,
                                                     const int* __restrict__ glist, const Work& W, const StageCfg& S,
                                                     Scalars* sc, int ntx, int tile) {
    pdl_wait();
    const bool stop = halted(sc);
    constexpr int NS = (NB == 1) ? 1 : (NB == 5 ? 8 : 7);
    constexpr int SR = sums_stride(NS);
    static_assert(SR <= SUMS_MAX, "reduced sums overflow");
    __shared__ TileHdr T;
    extern __shared__ double smem_raw[];
    const SmemView SM = smem_view<NB == 5>(smem_raw, P.cap);
    const int tx = tile % ntx, ty = tile / ntx;
    stage_halo<false, NB == 5>(P, cur, Lc, gstart, glist, tx * TX - 1, ty * TY - 1, T, SM);
    pdl_release();
    if (stop) return;
    const int n_own = T.own_off[OC];
    const int lane = threadIdx.x & (G - 1);
    const bool sum_model = P.sph_model == 1;
    const bool early = S.mode == MODE_STAGE;
    auto own = [&](int o, int& i, double& x, double& y, double& u, double& v) {
        const int ki = SM.own_k[o];
        i = SM.idx[ki];
        x = SM.x[ki];
        y = SM.y[ki];
        u = SM.u[ki];
        v = NB >= 4 ? SM.v[ki] : 0.0;
    };
    for (int ob = 0; ob < n_own; ob += PPB) {
        {
            const int slot = (int)threadIdx.x / G;
            const int o = ob + slot;
            const bool active = o < n_own;
            int ki = 0, hc = 0;
            if (active) { ki = SM.own_k[o]; hc = SM.own_hc[o]; }
            const double my_x = SM.x[ki], my_y = SM.y[ki], my_u = SM.u[ki];
            double my_v = 0, my_rho = 0, my_pre = 0, my_tem = 0;
            if constexpr (NB >= 4) { my_v = SM.v[ki]; my_rho = SM.rho[ki]; my_pre = SM.pre[ki]; }
            if constexpr (NB == 5) my_tem = SM.tem[ki];
            double acc[NS];
#pragma unroll
            for (int k = 0; k < NS; ++k) acc[k] = 0.0;
            tile_pairs<G>(T, SM, active, hc, lane, ki, my_x, my_y, P.h_eff_sq, [&](int k) {
                const double x_ij = my_x - SM.x[k], y_ij = my_y - SM.y[k];
                const double r = sqrt(x_ij * x_ij + y_ij * y_ij);
                const double dW = dev_dW<double>(P.kt, r, P.ih1, P.m3h, P.m5h, P.wnorm);
                const double Vj = SM.vol[k];
                const double L = ((2.0 * Vj) * dW) / r;
                if constexpr (NB == 1) {
                    acc[0] = fma(L, my_u - SM.u[k], acc[0]);
                } else {
                    const double gx = ((dW * x_ij) / r) * Vj, gy = ((dW * y_ij) / r) * Vj;
                    acc[0] = fma(gx, SM.u[k] - my_u, acc[0]);
                    acc[1] = fma(gy, SM.v[k] - my_v, acc[1]);
                    const double pj = SM.pre[k];
                    const double dp = sum_model ? pj + my_pre : pj - my_pre;
                    acc[2] = fma(gx, dp, acc[2]);
                    acc[3] = fma(gy, dp, acc[3]);
                    acc[4] = fma(L, my_u - SM.u[k], acc[4]);
                    acc[5] = fma(L, my_v - SM.v[k], acc[5]);
                    if constexpr (NB == 5) acc[7] = fma(L, my_tem - SM.tem[k], acc[7]);
                    acc[6] = fma(L, my_rho - SM.rho[k], acc[6]);
                }
            });
            group_reduce<G>(acc);
            if (active && lane == 0) {
                double* sm = SM.sums + slot * SR;
#pragma unroll
                for (int k = 0; k < NS; ++k) sm[k] = acc[k];
            }
        }
        __syncthreads();
        double red = 0.0;
        const int o = ob + (int)threadIdx.x;
        if ((int)threadIdx.x < PPB && o < n_own) {
            const double* sm = SM.sums + threadIdx.x * SR;
            const int ki = SM.own_k[o];
            double my_v = 0, my_rho = 0, my_tem = 0;
            if constexpr (NB >= 4) { my_v = SM.v[ki]; my_rho = SM.rho[ki]; }
            if constexpr (NB == 5) my_tem = SM.tem[ki];
            const int i = SM.idx[ki];
            double Ru, Rv, Rr, Rt;
            rhs_classical<NB>(P, W, i, my_rho, my_tem, sm, Ru, Rv, Rr, Rt);
            keep_rhs<NB>(W, S, i, Ru, Rv, Rr, Rt);
            if (early) {
                const OldFields of = load_old_fields<NB>(P, W, S, i, SM.u[ki], my_v, my_rho, my_tem);
                red = stage_fields<NB>(P, nxt, W, S, sc, i, my_v, my_rho, my_tem, Ru, Rv, Rr, Rt, of);
            }
        } else if (G > 1 && early && ob == 0 && (int)threadIdx.x >= PPB) {
            // the warps idle while the RHS is formed move the own particles
            stage_move_own<NB>(P, nxt, Ln, gstart, W, S, sc, n_own, (int)threadIdx.x - PPB, blockDim.x - PPB, own);
        }
        if (S.mode == MODE_STAGE && S.last && (S.do_umax || S.do_steady))
            warp_max_atomic(S.do_umax ? &sc->umax2 : &sc->dfmax, red);
        __syncthreads();
    }
    if constexpr (G == 1)
        if (early) stage_move_own<NB>(P, nxt, Ln, gstart, W, S, sc, n_own, threadIdx.x, blockDim.x, own);
}

template <int NB, int G, int TIGHT = 0>
__global__ void __launch_bounds__(PPB * G, tile_min_blocks(G, TIGHT))
    k_stage_classical(const Phys P, const Fld cur, const Fld nxt, const Lst Lc, const Lst Ln,
                      const int* __restrict__ gstart, const int* __restrict__ glist, const Work W, const StageCfg S,
                      Scalars* sc, int ntx, const int* __restrict__ tiles) {
    stage_body_classical<NB, G>(P, cur, nxt, Lc, Ln, gstart, glist, W, S, sc, ntx,
                                tiles ? tiles[blockIdx.x] : (int)blockIdx.x);
}

// MIXED: 0 FP64, 1 mixed precision, 2 mixed precision with compensated pair sums.
template <int NB, int G, int MIXED>
__device__ __forceinline__ void stage_body(const Phys& P, const Fld& cur, const Fld& nxt, const Lst& Lc, const Lst& Ln,
                                           const int* __restrict__ gstart, const int* __restrict__ glist,
                                           const Work& W, const StageCfg& S, Scalars* sc, int ntx, int tile) {
    if constexpr (MIXED != 0) stage_body_mx<NB, G, MIXED == 2>(P, cur, nxt, Lc, Ln, gstart, glist, W, S, sc, ntx, tile);
    else stage_body_fp64<NB, G>(P, cur, nxt, Lc, Ln, gstart, glist, W, S, sc, ntx, tile);
}

template <int NB, int G, int TIGHT = 0, int MIXED = 0>
__global__ void __launch_bounds__(PPB * G, tile_min_blocks(G, TIGHT))
    k_stage(const Phys P, const Fld cur, const Fld nxt, const Lst Lc, const Lst Ln, const int* __restrict__ gstart,
            const int* __restrict__ glist, const Work W, const StageCfg S, Scalars* sc, int ntx,
            const int* __restrict__ tiles) {   // tile of each CTA (NULL: CTA i runs tile i)
    stage_body<NB, G, MIXED>(P, cur, nxt, Lc, Ln, gstart, glist, W, S, sc, ntx, tiles ? tiles[blockIdx.x] : (int)blockIdx.x);
}

// =======================================================================================
// k_ghost: interpolation at the virtual markers + extrapolation to the ghost particles.
// WQ = 3 / 6: LS type B (interpolate_LSSPH_B_mod.f90, WALL_MODEL 2 / 3); WQ = 1: CSPH
// (interpolate_CSPH_mod.f90, WALL_MODEL 1).  NB = 1 (problem 1: u), 3 (u,v,p), 4 (+T).
// One CTA per chunk of at most PPB markers of one tile; also clears the scatter counters
// of the cell list the preceding stage consumed (zero_cnt) and, after PST, the U_max slot.
// =======================================================================================
struct VMTiles {
    const int* tile;    // [n] tile id of each chunk
    const int* start;   // [n+1] chunk ranges into vm
    const int* vm;      // virtual-marker ids grouped by tile, ascending
};

// One chunk (<= PPB markers of one tile) of one solve; nchunk = chunks of this solve.
template <int NB, int G, int WQ>
__device__ __forceinline__ void ghost_work(const Phys& P, const Fld& F, const Lst& L, const int* __restrict__ gstart,
                                           const int* __restrict__ glist, const VMd& V, const VMTiles& VT, int ntx,
                                           int* zero_cnt, int reset_umax, Scalars* sc, int chunk, int nchunk) {
    // a stopped solve (steady state, step budget, error) keeps its cell lists as they are,
    // so that it can resume exactly where it stopped
    pdl_wait();
    const bool stop = halted(sc);
    if (zero_cnt && !stop) {
        for (int c = chunk * blockDim.x + threadIdx.x; c < P.ncell; c += nchunk * blockDim.x) zero_cnt[c] = 0;
    }
    if (reset_umax && chunk == 0 && threadIdx.x == 0) sc->umax2 = 0ull;
    if (P.num_ext == 0) {   // periodic domain: no ghosts, only the bookkeeping above (one chunk)
        pdl_release();
        return;
    }
    constexpr int Q = (WQ == 1) ? 1 : WQ;
    constexpr int NU = Q * (Q + 1) / 2;
    __shared__ TileHdr T;
    extern __shared__ double smem_raw[];
    const SmemView SM = smem_view<NB == 4>(smem_raw, P.cap);
    const int tile = VT.tile[chunk];
    const int tx = tile % ntx, ty = tile / ntx;
    const int cx0 = tx * TX - 1, cy0 = ty * TY - 1;
    stage_halo<true, NB == 4>(P, F, L, gstart, glist, cx0, cy0, T, SM);
    pdl_release();
    if (stop) return;
    const int v0 = VT.start[chunk], nvm = VT.start[chunk + 1] - v0;
    const int lane = threadIdx.x & (G - 1);
    const int o = (int)threadIdx.x / G;
    const bool active = o < nvm;
    int me = 0, hc = 0;
    double my_x = 0, my_y = 0;
    if (active) {
        me = VT.vm[v0 + o];
        my_x = V.x[me];
        my_y = V.y[me];
        const int key = V.key[me];
        hc = (key % P.nx - cx0) + (key / P.nx - cy0) * HX;
    }
    double Mu[NU];
    double B[NB][Q];
    double sw = 0.0;
#pragma unroll
    for (int k = 0; k < NU; ++k) Mu[k] = 0.0;
#pragma unroll
    for (int c = 0; c < NB; ++c)
#pragma unroll
        for (int k = 0; k < Q; ++k) B[c][k] = 0.0;
    int cnt = 0;
    // the pair loop is compiled for the Wendland C2 kernel and for any type (as
    // stage_pair_sums), so that the loop holds no branch on the kernel type
    auto ls_pairs = [&](auto KTc) {
        constexpr int KT = decltype(KTc)::value;
        const int kt = KT ? KT : P.kt;
        cnt = tile_pairs<G>(T, SM, active, hc, lane, -1, my_x, my_y, P.h_eff_sq, [&](int k) {
            const double xji = SM.x[k] - my_x, yji = SM.y[k] - my_y;
            const double Wv = dev_W(kt, sqrt(xji * xji + yji * yji), P.ih1, P.wnorm);
            const double VW = SM.vol[k] * Wv;
            double a[Q];
            a[0] = 1.0;
            if constexpr (Q >= 3) {
                a[1 % Q] = xji * P.ih1;
                a[2 % Q] = yji * P.ih1;
            }
            if constexpr (Q == 6) {
                a[3] = ((xji * xji) * 0.5) * P.ih2B;
                a[4] = (xji * yji) * P.ih2B;
                a[5] = ((yji * yji) * 0.5) * P.ih2B;
            }
            double f[NB];
            f[0] = SM.u[k];
            if constexpr (NB >= 3) { f[1] = SM.v[k]; f[2] = SM.pre[k]; }
            if constexpr (NB == 4) f[3] = SM.tem[k];
#pragma unroll
            for (int ii = 0; ii < Q; ++ii) {
                const double VWa = VW * a[ii];
#pragma unroll
                for (int c = 0; c < NB; ++c) B[c][ii] = fma(VWa, f[c], B[c][ii]);
#pragma unroll
                for (int jj = 0; jj <= ii; ++jj) Mu[UT(jj, ii)] = fma(VWa, a[jj], Mu[UT(jj, ii)]);
            }
        });
    };
    if constexpr (WQ != 1) {
        if (P.kt == 3) ls_pairs(std::integral_constant<int, 3>{});
        else ls_pairs(std::integral_constant<int, 0>{});
    }
    if (active && WQ == 1) {
        for_tile_candidates<G>(T, hc, lane, [&](int k) {
            if constexpr (WQ == 1) {
                const double xij = my_x - SM.x[k], yij = my_y - SM.y[k];
                const double r2 = xij * xij + yij * yij;
                if (r2 > P.h_eff_sq) return;
                const double Wv = dev_W(P.kt, sqrt(r2), P.ih1, P.wnorm);
                ++cnt;
                const double VW = SM.vol[k] * Wv;
                sw = sw + VW;
                B[0][0] = fma(VW, SM.u[k], B[0][0]);
                if constexpr (NB >= 3) {
                    B[1][0] = fma(VW, SM.v[k], B[1][0]);
                    B[2][0] = fma(VW, SM.pre[k], B[2][0]);
                }
                if constexpr (NB == 4) B[3][0] = fma(VW, SM.tem[k], B[3][0]);
            }
        });
    }
    group_reduce<G>(Mu);
#pragma unroll
    for (int c = 0; c < NB; ++c) group_reduce<G>(B[c]);
    if constexpr (G > 1) {
        sw = group_sum<G>(sw);
        if (WQ == 1) cnt = group_sum_i<G>(cnt);   // tile_pairs already returns the group total
    }
    if (!active || lane != 0) return;

    double val[4] = {0.0, 0.0, 0.0, 0.0};
    if constexpr (WQ == 1) {
        if (cnt > 0 && sw > 1.0e-12) {
#pragma unroll
            for (int c = 0; c < NB; ++c) val[c] = B[c][0] / sw;
        }
    } else {
        if (cnt >= Q) {
            double A[Q][Q];
#pragma unroll
            for (int r = 0; r < Q; ++r)
#pragma unroll
                for (int c = 0; c < Q; ++c) A[r][c] = (r <= c) ? Mu[UT(r, c)] : Mu[UT(c, r)];
            if (!lu_solve<Q, NB>(A, B)) atomicOr(&sc->warn, WARN_SINGULAR);
#pragma unroll
            for (int c = 0; c < NB; ++c) val[c] = B[c][0];
        }
    }
    const int you = P.num_int + me;
    if constexpr (NB == 1) {   // extrapolate_diff_test_mod.f90:40-103
        const double vu = val[0];
        const int md = V.mode[me];
        const double K = V.K[me];
        double ug;
        if (md == XM_COPY) ug = vu;
        else if (md == XM_K_MINUS) ug = K - vu;
        else if (md == XM_PLUS_K) ug = vu + K;
        else ug = -vu;
        V.u[me] = vu;
        F.u[you] = ug;
    } else {                   // extrapolate_VM_to_WL_mod.f90:40-271
        const double vu = val[0], vv = val[1], vp = val[2], vt = val[3];
        V.u[me] = vu; V.v[me] = vv; V.pre[me] = vp;
        if constexpr (NB == 4) V.tem[me] = vt;
        const double nx = V.nx[me], ny = V.ny[me];
        const int t = V.ptype[me];
        int ubc = 2, tbc = 0;
        double Tw = 0.0, hydro = 0.0;
        bool hyd = false;
        if (t == 1) { ubc = P.u_bc_bottom; tbc = P.tem_bc_bottom; Tw = P.tem_bottom; hyd = true; hydro = P.hydro_coef_bottom; }
        else if (t == 2) { ubc = P.u_bc_top; tbc = P.tem_bc_top; Tw = P.tem_top; hyd = true; hydro = P.hydro_coef_top; }
        else if (t == 3) { ubc = P.u_bc_left; tbc = P.tem_bc_left; Tw = P.tem_left; }
        else if (t == 4) { ubc = P.u_bc_right; tbc = P.tem_bc_right; Tw = P.tem_right; }
        else if (t == 5 || t == 6) { ubc = 2; tbc = P.tem_bc_bottom; Tw = P.tem_bottom; hyd = true; hydro = P.hydro_coef_bottom; }
        else { ubc = (P.u_bc_top == 3) ? 3 : 2; tbc = P.tem_bc_top; Tw = P.tem_top; hyd = true; hydro = P.hydro_coef_top; }
        double ug, vg;
        if (ubc == 1) {
            const double u_n = vu * nx + vv * ny;
            ug = vu - (2.0 * u_n) * nx;
            vg = vv - (2.0 * u_n) * ny;
        } else if (ubc == 3) {
            ug = 2.0 * P.u_top - vu;
            vg = -vv;
        } else {
            ug = -vu;
            vg = -vv;
        }
        double pg = vp;
        if constexpr (NB == 4) {
            if (hyd && tbc == 1) pg = vp + hydro * (F.y[you] - my_y);
        }
        F.u[you] = ug; F.v[you] = vg; F.pre[you] = pg;
        if constexpr (NB == 4) F.tem[you] = (tbc == 1) ? 2.0 * Tw - vt : vt;
    }
}

// reset_umax marks the ghost launch that ends a time step (after PST).
template <int NB, int G, int WQ>
__device__ __forceinline__ void ghost_body(const Phys& P, const Fld& F, const Lst& L, const int* __restrict__ gstart,
                                           const int* __restrict__ glist, const VMd& V, const VMTiles& VT, int ntx,
                                           int* zero_cnt, int reset_umax, Scalars* sc, int chunk, int nchunk) {
    ghost_work<NB, G, WQ>(P, F, L, gstart, glist, V, VT, ntx, zero_cnt, reset_umax, sc, chunk, nchunk);
    if (reset_umax) end_of_step(sc, nchunk);
}

template <int NB, int G, int WQ>
__global__ void __launch_bounds__(PPB * G) k_ghost(const Phys P, const Fld F, const Lst L,
                                                   const int* __restrict__ gstart, const int* __restrict__ glist,
                                                   const VMd V, const VMTiles VT, int ntx, int* zero_cnt,
                                                   int reset_umax, Scalars* sc) {
    ghost_body<NB, G, WQ>(P, F, L, gstart, glist, V, VT, ntx, zero_cnt, reset_umax, sc, blockIdx.x, gridDim.x);
}

// =======================================================================================
// k_pst: particle shifting (q = 5) + copy-back + EOS + cell scatter.
// NB = 3 (u,v,rho) or 4 (+T).  umax2 holds max(u^2+v^2) of the state being shifted.
// =======================================================================================
// Shifted position of the own particle at staged position ki, its cell key, and its entry
// in the next cell list (PST_mod.f90:85-113 with update_cell).
__device__ __forceinline__ void pst_move(const Phys& P, const Fld& nxt, const Lst& Ln, const int* __restrict__ gstart,
                                         const Work& W, Scalars* sc, const SmemView& SM, int ki, double dx,
                                         double dy) {
    const int i = SM.idx[ki];
    double xn = SM.x[ki] + dx, yn = SM.y[ki] + dy;
    if (P.periodic) { xn = wrap_pos(xn, P.Lx); yn = wrap_pos(yn, P.Lx); }
    nxt.x[i] = xn;
    nxt.y[i] = yn;
    if (!(isfinite(xn) && isfinite(yn))) atomicOr(&sc->err, ERR_NONFINITE);
    const int nk = cell_key_mul(P, xn, yn, sc);
    if (nk >= 0) {
        W.key[i] = nk;
        if (P.split_pos) put_split_pos(P, nxt, i, xn, yn, nk);
    }
    scatter_to_cell(P, Ln, gstart, nk, i, sc);
}

// FP64 pair phase of one own particle of PST (shift_interpolate_mod.f90:120-190): the LS
// moment matrix and b vectors of the fields to interpolate (Md, Bd) and the shift sums
// sum (1 + 0.2 (W/W_ave)^4) V_j grad W (sd), combined over the particle's G lanes.  Returns
// the in-radius count.  K: order of the Taylor basis (2: q = 5 for SPH_MODEL 3; 1: q = 2
// for the classical models).  Shared by the fused PST kernel and the split pair kernel.
template <int NB, int G, int K, int KT>
__device__ __forceinline__ int pst_pair_sums_kt(const Phys& P, const TileHdr& T, const SmemView& SM, bool active,
                                                int ki, int hc, int lane,
                                                double (&Md)[((K == 1) ? 2 : 5) * (((K == 1) ? 2 : 5) + 1) / 2],
                                                double (&Bd)[NB][(K == 1) ? 2 : 5], double (&sd)[2]) {
    const int kt = KT ? KT : P.kt;
    constexpr int Q = (K == 1) ? 2 : 5;
    constexpr int QU = Q * (Q + 1) / 2;
    const double my_x = SM.x[ki], my_y = SM.y[ki], my_u = SM.u[ki], my_v = SM.v[ki], my_rho = SM.rho[ki];
    double my_tem = 0.0;
    if constexpr (NB == 4) my_tem = SM.tem[ki];
    using R = double;
    const PairConst<R> C(P);
    R Mu[QU];
    R B[NB][Q];
#pragma unroll
    for (int k = 0; k < QU; ++k) Mu[k] = R(0);
#pragma unroll
    for (int c = 0; c < NB; ++c)
#pragma unroll
        for (int k = 0; k < Q; ++k) B[c][k] = R(0);
    R sxy[2] = {R(0), R(0)};
    const int cnt = tile_pairs<G>(T, SM, active, hc, lane, ki, my_x, my_y, P.h_eff_sq, [&](int k) {
        const R xji = R(SM.x[k] - my_x);
        const R yji = R(SM.y[k] - my_y);
        const R r = sqrt(xji * xji + yji * yji);
        const R Wv = dev_W<R>(kt, r, C.ih1, C.wnorm);
        const R dWdr = dev_dW<R>(kt, r, C.ih1, C.m3h, C.m5h, C.wnorm);
        const R Vj = R(SM.vol[k]);
        const R VW = Vj * Wv;
        const R rinv = R(1) / r;
        const R gx = ((dWdr * (-xji)) * rinv) * Vj;
        const R gy = ((dWdr * (-yji)) * rinv) * Vj;
        const R t = Wv * C.iWave, t2 = t * t, t4 = t2 * t2;
        const R fac = R(1.0) + R(0.2) * t4;
        sxy[0] = fma(fac, gx, sxy[0]);
        sxy[1] = fma(fac, gy, sxy[1]);
        R a[Q];
        basis_A<R>(C.ih1, C.ih2A, xji, yji, a);
        R df[NB];
        df[0] = R(SM.u[k] - my_u);
        df[1] = R(SM.v[k] - my_v);
        df[2] = R(SM.rho[k] - my_rho);
        if constexpr (NB == 4) df[3] = R(SM.tem[k] - my_tem);
        accumulate_A<NB, R>(Mu, B, VW, a, df);
    });
    group_reduce_to<G>(Mu, Md);
#pragma unroll
    for (int c = 0; c < NB; ++c) group_reduce_to<G>(B[c], Bd[c]);
    group_reduce_to<G>(sxy, sd);
    return cnt;
}

// Compiled for the Wendland C2 kernel and for any type, as stage_pair_sums.
template <int NB, int G, int K>
__device__ __forceinline__ int pst_pair_sums(const Phys& P, const TileHdr& T, const SmemView& SM, bool active,
                                             int ki, int hc, int lane,
                                             double (&Md)[((K == 1) ? 2 : 5) * (((K == 1) ? 2 : 5) + 1) / 2],
                                             double (&Bd)[NB][(K == 1) ? 2 : 5], double (&sd)[2]) {
    if (P.kt == 3) return pst_pair_sums_kt<NB, G, K, 3>(P, T, SM, active, ki, hc, lane, Md, Bd, sd);
    return pst_pair_sums_kt<NB, G, K, 0>(P, T, SM, active, ki, hc, lane, Md, Bd, sd);
}

template <int NB, int G, int K = 2>
__device__ __forceinline__ void pst_body_fp64(const Phys& P, const Fld& cur, const Fld& nxt, const Lst& Lc, const Lst& Ln,
                                         const int* __restrict__ gstart, const int* __restrict__ glist, const Work& W,
                                         Scalars* sc, int ntx, int tile) {
    pdl_wait();
    const bool stop = halted(sc);   // consumed after staging, so its load overlaps the staging loads
    constexpr int Q = (K == 1) ? 2 : 5;
    constexpr int QU = Q * (Q + 1) / 2;
    constexpr int SR = sums_stride(QU + Q * NB + 3);
    static_assert(SR <= SUMS_MAX, "reduced sums overflow");
    __shared__ TileHdr T;
    extern __shared__ double smem_raw[];
    const SmemView SM = smem_view<NB == 4>(smem_raw, P.cap);
    const int tx = tile % ntx, ty = tile / ntx;
    stage_halo<false, NB == 4>(P, cur, Lc, gstart, glist, tx * TX - 1, ty * TY - 1, T, SM);
    pdl_release();
    if (stop) return;
    const int n_own = T.own_off[OC];
    const double U_max = sqrt(__longlong_as_double((long long)sc->umax2));
    const double coe = ((P.PST_c * U_max) * P.dt) * P.h;
    const int lane = threadIdx.x & (G - 1);
    for (int ob = 0; ob < n_own; ob += PPB) {
        {
            const int slot = (int)threadIdx.x / G;
            const int o = ob + slot;
            const bool active = o < n_own;
            int ki = 0, hc = 0;
            if (active) { ki = SM.own_k[o]; hc = SM.own_hc[o]; }
            double Md[QU], Bd[NB][Q], sd[2];
            const int cnt = pst_pair_sums<NB, G, K>(P, T, SM, active, ki, hc, lane, Md, Bd, sd);
            if (active && lane == 0) {
                double* sm = SM.sums + slot * SR;
#pragma unroll
                for (int k = 0; k < QU; ++k) sm[k] = Md[k];
#pragma unroll
                for (int c = 0; c < NB; ++c)
#pragma unroll
                    for (int k = 0; k < Q; ++k) sm[QU + Q * c + k] = Bd[c][k];
                sm[SR - 3] = sd[0];
                sm[SR - 2] = sd[1];
                sm[SR - 1] = (double)cnt;
            }
        }
        __syncthreads();
        const int o = ob + (int)threadIdx.x;
        // shift vector of pass slot t, clamped to 0.2 h (shift_interpolate_mod.f90:216-225)
        auto shift = [&](int t, double& dx, double& dy) {
            const double* sm = SM.sums + t * SR;
            dx = -coe * sm[SR - 3];
            dy = -coe * sm[SR - 2];
            const double rr = sqrt(dx * dx + dy * dy);
            if (rr > 0.2 * P.h) {
                dx = ((0.2 * P.h) * dx) / rr;
                dy = ((0.2 * P.h) * dy) / rr;
            }
        };
        // with more than one warp, the warps idle in the solve move this pass's particles,
        // key them and append them to the next cell list (the shift needs no solve)
        constexpr bool split = G > 1;
        if ((int)threadIdx.x < PPB && o < n_own) {
            const double* sm = SM.sums + threadIdx.x * SR;
            const int ki = SM.own_k[o];
            const int cnt = (int)sm[SR - 1];
            double dx, dy;
            shift(threadIdx.x, dx, dy);
            double B[NB][Q];
            {
                double A[Q][Q];
#pragma unroll
                for (int r = 0; r < Q; ++r)
#pragma unroll
                    for (int c = 0; c < Q; ++c) A[r][c] = (r <= c) ? sm[UT(r, c)] : sm[UT(c, r)];
#pragma unroll
                for (int c = 0; c < NB; ++c)
#pragma unroll
                    for (int k = 0; k < Q; ++k) B[c][k] = sm[QU + Q * c + k];
                if (cnt >= Q) {
                    if (!lu_solve<Q, NB>(A, B)) atomicOr(&sc->warn, WARN_SINGULAR);
                } else {
#pragma unroll
                    for (int c = 0; c < NB; ++c)
#pragma unroll
                        for (int k = 0; k < Q; ++k) B[c][k] = 0.0;
                }
            }
            // interpolation a(dr) . d (shift_interpolate_mod.f90:255-298)
            double a[Q];
            basis_A(P, dx, dy, a);
            double acc[NB];
#pragma unroll
            for (int c = 0; c < NB; ++c) {
                double sacc = 0.0;
#pragma unroll
                for (int k = 0; k < Q; ++k) sacc = fma(a[k], B[c][k], sacc);
                acc[c] = sacc;
            }
            const int i = SM.idx[ki];
            const double un = SM.u[ki] + acc[0], vn = SM.v[ki] + acc[1], rn = SM.rho[ki] + acc[2];
            nxt.u[i] = un; nxt.v[i] = vn; nxt.rho[i] = rn;
            nxt.pre[i] = P.c_sq * (rn - P.rho_ref);
            nxt.vol[i] = P.SP_mass / rn;
            bool finite = isfinite(un) && isfinite(vn) && isfinite(rn);
            if constexpr (NB == 4) { const double tn = SM.tem[ki] + acc[3]; nxt.tem[i] = tn; finite = finite && isfinite(tn); }
            if (!finite) atomicOr(&sc->err, ERR_NONFINITE);
            if (!split) pst_move(P, nxt, Ln, gstart, W, sc, SM, ki, dx, dy);
        } else if (split && (int)threadIdx.x >= PPB) {
            for (int t = (int)threadIdx.x - PPB; t < PPB && ob + t < n_own; t += blockDim.x - PPB) {
                double dx, dy;
                shift(t, dx, dy);
                pst_move(P, nxt, Ln, gstart, W, sc, SM, SM.own_k[ob + t], dx, dy);
            }
        }
        __syncthreads();
    }
}


// Mixed-precision PST: FP32 staging and pair phase, FP64 solve (COMP: compensated sums and
// one refinement step) and update.
template <int NB, int G, bool COMP>
__device__ __forceinline__ void pst_body_mx(const Phys& P, const Fld& cur, const Fld& nxt, const Lst& Lc,
                                            const Lst& Ln, const int* __restrict__ gstart,
                                            const int* __restrict__ glist, const Work& W, Scalars* sc, int ntx,
                                            int tile) {
    pdl_wait();
    const bool stop = halted(sc);
    constexpr int Q = 5;
    constexpr int SR = sums_stride(15 + 5 * NB + 3);
    static_assert(SR <= SUMS_MAX, "reduced sums overflow");
    __shared__ TileHdr T;
    extern __shared__ double smem_raw[];
    const SmemMx SM = smem_view_mx<NB == 4>(smem_raw, P.cap);
    const int tx = tile % ntx, ty = tile / ntx;
    const int cx0 = tx * TX - 1, cy0 = ty * TY - 1;
    stage_lists<false>(P, Lc, gstart, glist, cx0, cy0, T, SM);
    stage_fields_mx<NB == 4>(P, cur, cx0, cy0, T, SM);
    pdl_release();
    if (stop) return;
    const int n_own = T.own_off[OC];
    const double U_max = sqrt(__longlong_as_double((long long)sc->umax2));
    const double coe = ((P.PST_c * U_max) * P.dt) * P.h;
    const int lane = threadIdx.x & (G - 1);
    for (int ob = 0; ob < n_own; ob += PPB) {
        {
            const int slot = (int)threadIdx.x / G;
            const int o = ob + slot;
            const bool active = o < n_own;
            int ki = 0, hc = 0;
            if (active) { ki = SM.own_k[o]; hc = SM.own_hc[o]; }
            double Md[15], Bd[NB][Q], sd[2];
            const int cnt = mx_pair_sums<NB, G, COMP, true>(P, T, SM, active, ki, hc, lane, Md, Bd, sd);
            if (active && lane == 0) {
                double* sm = SM.sums + slot * SR;
#pragma unroll
                for (int k = 0; k < 15; ++k) sm[k] = Md[k];
#pragma unroll
                for (int c = 0; c < NB; ++c)
#pragma unroll
                    for (int k = 0; k < Q; ++k) sm[15 + 5 * c + k] = Bd[c][k];
                sm[SR - 3] = sd[0];
                sm[SR - 2] = sd[1];
                sm[SR - 1] = (double)cnt;
            }
        }
        __syncthreads();
        const int o = ob + (int)threadIdx.x;
        if ((int)threadIdx.x < PPB && o < n_own) {
            double* sm = SM.sums + threadIdx.x * SR;
            const int i = SM.idx[SM.own_k[o]];
            const double my_x = cur.x[i], my_y = cur.y[i], my_u = cur.u[i], my_v = cur.v[i], my_rho = cur.rho[i];
            double my_tem = 0.0;
            if constexpr (NB == 4) my_tem = cur.tem[i];
            // shift vector, clamped to 0.2 h (shift_interpolate_mod.f90:216-225)
            double dx = -coe * sm[SR - 3], dy = -coe * sm[SR - 2];
            const double rr = sqrt(dx * dx + dy * dy);
            if (rr > 0.2 * P.h) {
                dx = ((0.2 * P.h) * dx) / rr;
                dy = ((0.2 * P.h) * dy) / rr;
            }
            if constexpr (COMP) solve_row_refined<Q, NB, false>(P, sm, (int)sm[SR - 1], sc);
            else solve_row_plain<Q, NB, false>(P, sm, (int)sm[SR - 1], sc);
            // interpolation a(dr) . d (shift_interpolate_mod.f90:255-298)
            double a[Q];
            basis_A(P, dx, dy, a);
            double acc[NB];
#pragma unroll
            for (int c = 0; c < NB; ++c) {
                double sacc = 0.0;
#pragma unroll
                for (int k = 0; k < Q; ++k) sacc = fma(a[k], sm[15 + 5 * c + k], sacc);
                acc[c] = sacc;
            }
            double xn = my_x + dx, yn = my_y + dy;
            if (P.periodic) { xn = wrap_pos(xn, P.Lx); yn = wrap_pos(yn, P.Lx); }
            const double un = my_u + acc[0], vn = my_v + acc[1], rn = my_rho + acc[2];
            nxt.x[i] = xn; nxt.y[i] = yn; nxt.u[i] = un; nxt.v[i] = vn; nxt.rho[i] = rn;
            nxt.pre[i] = P.c_sq * (rn - P.rho_ref);
            nxt.vol[i] = P.SP_mass / rn;
            bool finite = isfinite(xn) && isfinite(yn) && isfinite(un) && isfinite(vn) && isfinite(rn);
            if constexpr (NB == 4) { const double tn = my_tem + acc[3]; nxt.tem[i] = tn; finite = finite && isfinite(tn); }
            if (!finite) atomicOr(&sc->err, ERR_NONFINITE);
            const int nk = cell_key_mul(P, xn, yn, sc);
            if (nk >= 0) {
                W.key[i] = nk;
                if (P.split_pos) put_split_pos(P, nxt, i, xn, yn, nk);
            }
            scatter_to_cell(P, Ln, gstart, nk, i, sc);
        }
        __syncthreads();
    }
}

template <int NB, int G, int MIXED, int K = 2>
__device__ __forceinline__ void pst_body(const Phys& P, const Fld& cur, const Fld& nxt, const Lst& Lc, const Lst& Ln,
                                         const int* __restrict__ gstart, const int* __restrict__ glist, const Work& W,
                                         Scalars* sc, int ntx, int tile) {
    static_assert(!(MIXED != 0 && K != 2), "mixed precision runs the q = 5 basis only");
    if constexpr (MIXED != 0) pst_body_mx<NB, G, MIXED == 2>(P, cur, nxt, Lc, Ln, gstart, glist, W, sc, ntx, tile);
    else pst_body_fp64<NB, G, K>(P, cur, nxt, Lc, Ln, gstart, glist, W, sc, ntx, tile);
}

template <int NB, int G, int TIGHT = 0, int MIXED = 0, int K = 2>
__global__ void __launch_bounds__(PPB * G, tile_min_blocks(G, TIGHT))
    k_pst(const Phys P, const Fld cur, const Fld nxt, const Lst Lc, const Lst Ln, const int* __restrict__ gstart,
          const int* __restrict__ glist, const Work W, Scalars* sc, int ntx, const int* __restrict__ tiles) {
    pst_body<NB, G, MIXED, K>(P, cur, nxt, Lc, Ln, gstart, glist, W, sc, ntx, tiles ? tiles[blockIdx.x] : (int)blockIdx.x);
}

// =======================================================================================
// Batched kernels: one launch runs a phase for every solve of a batch.  Each CTA reads
// its (solve, tile-or-chunk) from a map built on the host and that solve's descriptor;
// buffer parities are the solve's base parity xor the launch's parity, so solves that
// joined the batch at different times keep their own ping-pong state.
// =======================================================================================
// =======================================================================================
// Mixed precision, split shape.  The fused mixed kernels run the FP64 LS solve in the same
// CTA as the FP32 pair phase, so the solve's registers and the shared-memory rows that hand
// the sums to it set the occupancy of the whole kernel, and three of a CTA's four warps wait
// at a barrier while one solves.  The split shape runs
//   k_stage_mxp / k_pst_mxp   tile staging + FP32 pair phase; each particle's reduced sums
//                             go to Work::sums (no solve, no barrier after the staging)
//   k_stage_solve / k_pst_solve   one thread per interior particle: FP64 factorisation (the
//                             compensated mode: plus one refinement step), RHS, RK update,
//                             cell key and scatter (PST: shift, interpolation, move)
// with the same arithmetic per particle as the fused kernels, so both shapes give identical
// bits and the autotuner may pick either.
// =======================================================================================
constexpr int MXS_ENTRIES = 15 + 5 * 5 + 1;   // the widest row: stage with temperature (41)
static_assert(15 + 5 * 4 + 3 <= MXS_ENTRIES, "PST rows fit");

// Pair phase of one tile (stage, or PST with its shift sums), sums to Work::sums.
template <int NB, int G, bool COMP, bool PST>
__device__ __forceinline__ void pairs_mx(const Phys& P, const Fld& cur, const Lst& Lc, const int* __restrict__ gstart,
                                         const int* __restrict__ glist, const Work& W, Scalars* sc, int ntx, int tile) {
    constexpr bool TEM = PST ? (NB == 4) : (NB == 5);
    constexpr int Q = 5;
    constexpr int NR = 15 + 5 * NB + (PST ? 2 : 0);   // then the neighbour count
    pdl_wait();
    bool stop = halted(sc);
    __shared__ TileHdr T;
    extern __shared__ double smem_raw[];
    const SmemMx SM = smem_view_mx_at<TEM>(nullptr, reinterpret_cast<float*>(smem_raw), P.cap);
    const int tx = tile % ntx, ty = tile / ntx;
    const int cx0 = tx * TX - 1, cy0 = ty * TY - 1;
    stage_lists<false>(P, Lc, gstart, glist, cx0, cy0, T, SM);
    stage_fields_mx<TEM>(P, cur, cx0, cy0, T, SM);
    pdl_release();
    // one decision per warp: the shuffles below need every lane of it
    if (__any_sync(0xffffffffu, stop)) return;
    const int n_own = T.own_off[OC];
    const int lane = threadIdx.x & (G - 1);
    const size_t N = (size_t)P.num_int;
    for (int ob = 0; ob < n_own; ob += PPB) {
        const int slot = (int)threadIdx.x / G;
        const int o = ob + slot;
        const bool active = o < n_own;
        int ki = 0, hc = 0;
        if (active) { ki = SM.own_k[o]; hc = SM.own_hc[o]; }
        double Md[15], Bd[NB][Q], sd[2] = {0.0, 0.0};
        const int cnt = mx_pair_sums<NB, G, COMP, PST>(P, T, SM, active, ki, hc, lane, Md, Bd, sd);
        if (active) {   // lane l of the particle's G stores entries l, l + G, ...
            const int i = SM.idx[ki];
            double* dst = W.sums + i;
#pragma unroll
            for (int e = 0; e <= NR; ++e) {
                if ((e & (G - 1)) != lane) continue;
                double val;
                if (e < 15) val = Md[e];
                else if (e < 15 + 5 * NB) val = Bd[(e - 15) / 5][(e - 15) % 5];
                else if (e < NR) val = sd[e - 15 - 5 * NB];
                else val = (double)cnt;
                dst[(size_t)e * N] = val;
            }
        }
    }
}

template <int NB, int G, int TIGHT, bool COMP>
__global__ void __launch_bounds__(PPB * G, tile_min_blocks(G, TIGHT))
    k_stage_mxp(const Phys P, const Fld cur, const Lst Lc, const int* __restrict__ gstart,
                const int* __restrict__ glist, const Work W, Scalars* sc, int ntx, const int* __restrict__ tiles) {
    pairs_mx<NB, G, COMP, false>(P, cur, Lc, gstart, glist, W, sc, ntx, tiles ? tiles[blockIdx.x] : (int)blockIdx.x);
}

template <int NB, int G, int TIGHT, bool COMP>
__global__ void __launch_bounds__(PPB * G, tile_min_blocks(G, TIGHT))
    k_pst_mxp(const Phys P, const Fld cur, const Lst Lc, const int* __restrict__ gstart,
              const int* __restrict__ glist, const Work W, Scalars* sc, int ntx, const int* __restrict__ tiles) {
    pairs_mx<NB, G, COMP, true>(P, cur, Lc, gstart, glist, W, sc, ntx, tiles ? tiles[blockIdx.x] : (int)blockIdx.x);
}

// Solve and update of the split shape, one thread per interior particle (the tail of the
// fused stage kernels: FP64 factorisation, RHS, RK update, key, scatter).  REF: one
// refinement step after the factorisation (the compensated mixed mode, as stage_body_mx with
// COMP); else the DGESV sequence of stage_body_fp64 and of the plain mixed mode.
template <int NB, bool REF>
__device__ __forceinline__ void stage_solve_row(const Phys& P, const Fld& cur, const Fld& nxt, const Lst& Ln,
                                               const int* __restrict__ gstart, const Work& W, const StageCfg& S,
                                               Scalars* sc, int i) {
    pdl_wait();
    pdl_release();
    if (__any_sync(0xffffffffu, halted(sc))) return;   // one decision per warp (warp_max_atomic)
    constexpr int Q = 5;
    constexpr int NR = 15 + 5 * NB;
    double red = 0.0;
    if (i < P.num_int) {
        const size_t N = (size_t)P.num_int;
        double row[NR];
#pragma unroll
        for (int e = 0; e < NR; ++e) row[e] = W.sums[(size_t)e * N + i];
        const int cnt = (int)W.sums[(size_t)NR * N + i];
        const double my_x = cur.x[i], my_y = cur.y[i], my_u = cur.u[i];
        double my_v = 0.0, my_rho = 0.0, my_tem = 0.0;
        if constexpr (NB >= 4) { my_v = cur.v[i]; my_rho = cur.rho[i]; }
        if constexpr (NB == 5) my_tem = cur.tem[i];
        if constexpr (REF) solve_row_refined<Q, NB, true>(P, row, cnt, sc);
        else solve_row_plain<Q, NB, true>(P, row, cnt, sc);
        double d[NB][Q];
#pragma unroll
        for (int c = 0; c < NB; ++c)
#pragma unroll
            for (int k = 0; k < Q; ++k) d[c][k] = row[15 + 5 * c + k];
        double Ru, Rv, Rr, Rt;
        rhs_ls<NB>(P, W, i, my_rho, my_tem, d, Ru, Rv, Rr, Rt);
        red = stage_advance<NB>(P, nxt, Ln, gstart, W, S, sc, i, my_x, my_y, my_u, my_v, my_rho, my_tem, Ru, Rv,
                                Rr, Rt);
    }
    if (S.mode == MODE_STAGE && S.last && (S.do_umax || S.do_steady))
        warp_max_atomic(S.do_umax ? &sc->umax2 : &sc->dfmax, red);
}

template <int NB, bool REF>
__global__ void __launch_bounds__(128) k_stage_solve(const Phys P, const Fld cur, const Fld nxt, const Lst Ln,
                                                     const int* __restrict__ gstart, const Work W, const StageCfg S,
                                                     Scalars* sc) {
    stage_solve_row<NB, REF>(P, cur, nxt, Ln, gstart, W, S, sc, (int)(blockIdx.x * blockDim.x + threadIdx.x));
}

// Shift, solve, interpolation and move of the split shape's PST, one thread per interior
// particle (the tail of pst_body_mx or of pst_body_fp64; REF as stage_solve_row).  NB = 3
// (u, v, rho) or 4 (+ T).
template <int NB, bool REF>
__device__ __forceinline__ void pst_solve_row(const Phys& P, const Fld& cur, const Fld& nxt, const Lst& Ln,
                                             const int* __restrict__ gstart, const Work& W, Scalars* sc, int i) {
    pdl_wait();
    pdl_release();
    if (halted(sc)) return;
    constexpr int Q = 5;
    constexpr int NR = 15 + 5 * NB;
    if (i >= P.num_int) return;
    const size_t N = (size_t)P.num_int;
    double row[NR];
#pragma unroll
    for (int e = 0; e < NR; ++e) row[e] = W.sums[(size_t)e * N + i];
    const double sx = W.sums[(size_t)NR * N + i], sy = W.sums[(size_t)(NR + 1) * N + i];
    const int cnt = (int)W.sums[(size_t)(NR + 2) * N + i];
    const double U_max = sqrt(__longlong_as_double((long long)sc->umax2));
    const double coe = ((P.PST_c * U_max) * P.dt) * P.h;
    const double my_x = cur.x[i], my_y = cur.y[i], my_u = cur.u[i], my_v = cur.v[i], my_rho = cur.rho[i];
    double my_tem = 0.0;
    if constexpr (NB == 4) my_tem = cur.tem[i];
    // shift vector, clamped to 0.2 h (shift_interpolate_mod.f90:216-225)
    double dx = -coe * sx, dy = -coe * sy;
    const double rr = sqrt(dx * dx + dy * dy);
    if (rr > 0.2 * P.h) {
        dx = ((0.2 * P.h) * dx) / rr;
        dy = ((0.2 * P.h) * dy) / rr;
    }
    if constexpr (REF) solve_row_refined<Q, NB, false>(P, row, cnt, sc);
    else solve_row_plain<Q, NB, false>(P, row, cnt, sc);
    // interpolation a(dr) . d (shift_interpolate_mod.f90:255-298)
    double a[Q];
    basis_A(P, dx, dy, a);
    double acc[NB];
#pragma unroll
    for (int c = 0; c < NB; ++c) {
        double sacc = 0.0;
#pragma unroll
        for (int k = 0; k < Q; ++k) sacc = fma(a[k], row[15 + 5 * c + k], sacc);
        acc[c] = sacc;
    }
    double xn = my_x + dx, yn = my_y + dy;
    if (P.periodic) { xn = wrap_pos(xn, P.Lx); yn = wrap_pos(yn, P.Lx); }
    const double un = my_u + acc[0], vn = my_v + acc[1], rn = my_rho + acc[2];
    nxt.x[i] = xn; nxt.y[i] = yn; nxt.u[i] = un; nxt.v[i] = vn; nxt.rho[i] = rn;
    nxt.pre[i] = P.c_sq * (rn - P.rho_ref);
    nxt.vol[i] = P.SP_mass / rn;
    bool finite = isfinite(xn) && isfinite(yn) && isfinite(un) && isfinite(vn) && isfinite(rn);
    if constexpr (NB == 4) { const double tn = my_tem + acc[3]; nxt.tem[i] = tn; finite = finite && isfinite(tn); }
    if (!finite) atomicOr(&sc->err, ERR_NONFINITE);
    const int nk = cell_key_mul(P, xn, yn, sc);
    if (nk >= 0) {
        W.key[i] = nk;
        if (P.split_pos) put_split_pos(P, nxt, i, xn, yn, nk);
    }
    scatter_to_cell(P, Ln, gstart, nk, i, sc);
}

template <int NB, bool REF>
__global__ void __launch_bounds__(128) k_pst_solve(const Phys P, const Fld cur, const Fld nxt, const Lst Ln,
                                                   const int* __restrict__ gstart, const Work W, Scalars* sc) {
    pst_solve_row<NB, REF>(P, cur, nxt, Ln, gstart, W, sc, (int)(blockIdx.x * blockDim.x + threadIdx.x));
}

// =======================================================================================
// FP64 split shape: the same two kernels in FP64.  The fused FP64 kernels hold the solve's
// registers and the sums rows in every CTA and idle three of four warps at a barrier during
// the solve; the pair kernel below stages the tile as they do, forms the same sums
// (stage_pair_sums / pst_pair_sums) and stores them to Work::sums in the layout pairs_mx
// uses, and k_stage_solve / k_pst_solve (REF = false) solve and update one particle per
// thread exactly as the fused FP64 kernels do.  Both shapes give identical bits.
// =======================================================================================
template <int NB, int G, bool PST>
__device__ __forceinline__ void pairs_fp(const Phys& P, const Fld& cur, const Lst& Lc, const int* __restrict__ gstart,
                                         const int* __restrict__ glist, const Work& W, Scalars* sc, int ntx, int tile) {
    constexpr bool TEM = PST ? (NB == 4) : (NB == 5);
    constexpr int Q = 5;
    constexpr int NR = 15 + 5 * NB + (PST ? 2 : 0);   // then the neighbour count
    pdl_wait();
    const bool stop = halted(sc);
    __shared__ TileHdr T;
    extern __shared__ double smem_raw[];
    const SmemView SM = smem_view<TEM>(smem_raw, P.cap, false);
    const int tx = tile % ntx, ty = tile / ntx;
    stage_halo<false, TEM>(P, cur, Lc, gstart, glist, tx * TX - 1, ty * TY - 1, T, SM);
    pdl_release();
    // one decision per warp: the shuffles below need every lane of it
    if (__any_sync(0xffffffffu, stop)) return;
    const int n_own = T.own_off[OC];
    const int lane = threadIdx.x & (G - 1);
    const size_t N = (size_t)P.num_int;
    for (int ob = 0; ob < n_own; ob += PPB) {
        const int slot = (int)threadIdx.x / G;
        const int o = ob + slot;
        const bool active = o < n_own;
        int ki = 0, hc = 0;
        if (active) { ki = SM.own_k[o]; hc = SM.own_hc[o]; }
        double Md[15], Bd[NB][Q], sd[2] = {0.0, 0.0};
        int cnt;
        if constexpr (PST) cnt = pst_pair_sums<NB, G, 2>(P, T, SM, active, ki, hc, lane, Md, Bd, sd);
        else cnt = stage_pair_sums<NB, G>(P, T, SM, active, ki, hc, lane, Md, Bd);
        if (active) {   // lane l of the particle's G stores entries l, l + G, ...
            const int i = SM.idx[ki];
            double* dst = W.sums + i;
#pragma unroll
            for (int e = 0; e <= NR; ++e) {
                if ((e & (G - 1)) != lane) continue;
                double val;
                if (e < 15) val = Md[e];
                else if (e < 15 + 5 * NB) val = Bd[(e - 15) / 5][(e - 15) % 5];
                else if (e < NR) val = sd[e - 15 - 5 * NB];
                else val = (double)cnt;
                dst[(size_t)e * N] = val;
            }
        }
    }
}

template <int NB, int G, int TIGHT>
__global__ void __launch_bounds__(PPB * G, tile_min_blocks(G, TIGHT))
    k_stage_fpp(const Phys P, const Fld cur, const Lst Lc, const int* __restrict__ gstart,
                const int* __restrict__ glist, const Work W, Scalars* sc, int ntx, const int* __restrict__ tiles) {
    pairs_fp<NB, G, false>(P, cur, Lc, gstart, glist, W, sc, ntx, tiles ? tiles[blockIdx.x] : (int)blockIdx.x);
}

template <int NB, int G, int TIGHT>
__global__ void __launch_bounds__(PPB * G, tile_min_blocks(G, TIGHT))
    k_pst_fpp(const Phys P, const Fld cur, const Lst Lc, const int* __restrict__ gstart,
              const int* __restrict__ glist, const Work W, Scalars* sc, int ntx, const int* __restrict__ tiles) {
    pairs_fp<NB, G, true>(P, cur, Lc, gstart, glist, W, sc, ntx, tiles ? tiles[blockIdx.x] : (int)blockIdx.x);
}

struct SolveDesc {
    Phys P;
    Fld F[2];
    Lst L[kLists];
    Work W;
    VMd V;
    VMTiles VT;
    const int* gstart;
    const int* glist;
    Scalars* sc;
    double dt1[4], dt2[4];     // per-stage RK step sizes (StageCfg.dt1/dt2 of a solo step)
    int ntx, sb, lb, nchunk;   // sb/lb: buffer parity of the solve when the descriptor was written
    int pad_;
};

struct BatchMap {
    const int2* cta;     // (solve, tile-or-chunk) per CTA
    const int* tstep;    // steps since the descriptors were written, mod 2 kLists (device)
    int sbf, lba;        // the group's state flip and list advance per step
};

// Buffer parity of a launch: the descriptor's, advanced by the steps taken since it was
// written, plus the launch's offset (ds, dl) from the start of the step.
__device__ __forceinline__ void batch_parity(const BatchMap& M, const SolveDesc& d, int ds, int dl, int& sb, int& lb) {
    const int t = *M.tstep;
    sb = d.sb ^ (M.sbf & t & 1) ^ ds;
    lb = (d.lb + M.lba * t + dl) % kLists;
}

// Copy the CTA's solve descriptor to shared memory (one global round trip for all of it).
__device__ __forceinline__ const SolveDesc& load_desc(const SolveDesc* D, int s, SolveDesc& sd) {
    static_assert(sizeof(SolveDesc) % 8 == 0, "descriptor is copied in 8-byte words");
    const unsigned long long* src = reinterpret_cast<const unsigned long long*>(D + s);
    unsigned long long* dst = reinterpret_cast<unsigned long long*>(&sd);
    for (int k = threadIdx.x; k < (int)(sizeof(SolveDesc) / 8); k += blockDim.x) dst[k] = src[k];
    __syncthreads();
    return sd;
}

template <int NB, int G, int TIGHT = 0, int MIXED = 0>
__global__ void __launch_bounds__(PPB * G, tile_min_blocks(G, TIGHT)) kb_stage(const SolveDesc* __restrict__ D, const BatchMap M, StageCfg S,
                                                    int ps, int pl) {
    __shared__ SolveDesc sd;
    const int2 m = M.cta[blockIdx.x];
    const SolveDesc& d = load_desc(D, m.x, sd);
    int sb, lb;
    batch_parity(M, d, ps, pl, sb, lb);
    S.dt1 = d.dt1[S.stage - 1];
    S.dt2 = d.dt2[S.stage - 1];
    stage_body<NB, G, MIXED>(d.P, d.F[sb], d.F[sb ^ 1], d.L[lb], d.L[next_list(lb)], d.gstart, d.glist, d.W, S, d.sc,
                             d.ntx, m.y);
}

template <int NB, int G, int WQ>
__global__ void __launch_bounds__(PPB * G) kb_ghost(const SolveDesc* __restrict__ D, const BatchMap M, int ps, int pl,
                                                    int zero_other, int reset_umax) {
    __shared__ SolveDesc sd;
    const int2 m = M.cta[blockIdx.x];
    const SolveDesc& d = load_desc(D, m.x, sd);
    int sb, lb;
    batch_parity(M, d, ps, pl, sb, lb);
    ghost_body<NB, G, WQ>(d.P, d.F[sb], d.L[lb], d.gstart, d.glist, d.V, d.VT, d.ntx,
                          zero_other ? d.L[prev_list(lb)].cnt : nullptr, reset_umax, d.sc, m.y, d.nchunk);
}

template <int NB, int G, int TIGHT = 0, int MIXED = 0>
__global__ void __launch_bounds__(PPB * G, tile_min_blocks(G, TIGHT)) kb_pst(const SolveDesc* __restrict__ D, const BatchMap M, int ps, int pl) {
    __shared__ SolveDesc sd;
    const int2 m = M.cta[blockIdx.x];
    const SolveDesc& d = load_desc(D, m.x, sd);
    int sb, lb;
    batch_parity(M, d, ps, pl, sb, lb);
    pst_body<NB, G, MIXED>(d.P, d.F[sb], d.F[sb ^ 1], d.L[lb], d.L[next_list(lb)], d.gstart, d.glist, d.W, d.sc,
                           d.ntx, m.y);
}

// Mixed precision, split shape, batched: the FP32 pair kernel over a group's (solve, tile) map
// (the solve kernel, kb_solve, follows the FP64 pair kernel below).
template <int NB, int G, int TIGHT, bool COMP, bool PST>
__global__ void __launch_bounds__(PPB * G, tile_min_blocks(G, TIGHT)) kb_pairs_mx(const SolveDesc* __restrict__ D,
                                                                                  const BatchMap M, int ps, int pl) {
    __shared__ SolveDesc sd;
    const int2 m = M.cta[blockIdx.x];
    const SolveDesc& d = load_desc(D, m.x, sd);
    int sb, lb;
    batch_parity(M, d, ps, pl, sb, lb);
    pairs_mx<NB, G, COMP, PST>(d.P, d.F[sb], d.L[lb], d.gstart, d.glist, d.W, d.sc, d.ntx, m.y);
}

// FP64 split shape, batched: the FP64 pair kernel over a group's (solve, tile) map.
template <int NB, int G, int TIGHT, bool PST>
__global__ void __launch_bounds__(PPB * G, tile_min_blocks(G, TIGHT)) kb_pairs_fp(const SolveDesc* __restrict__ D,
                                                                                  const BatchMap M, int ps, int pl) {
    __shared__ SolveDesc sd;
    const int2 m = M.cta[blockIdx.x];
    const SolveDesc& d = load_desc(D, m.x, sd);
    int sb, lb;
    batch_parity(M, d, ps, pl, sb, lb);
    pairs_fp<NB, G, PST>(d.P, d.F[sb], d.L[lb], d.gstart, d.glist, d.W, d.sc, d.ntx, m.y);
}

// The split shape's solve kernel over a group's (solve, block of 128 interior particles) map;
// REF as k_stage_solve.
template <int NB, bool PST, bool REF>
__global__ void __launch_bounds__(128) kb_solve(const SolveDesc* __restrict__ D, const BatchMap M, StageCfg S,
                                                   int ps, int pl) {
    __shared__ SolveDesc sd;
    const int2 m = M.cta[blockIdx.x];
    const SolveDesc& d = load_desc(D, m.x, sd);
    int sb, lb;
    batch_parity(M, d, ps, pl, sb, lb);
    const int i = m.y * 128 + (int)threadIdx.x;
    if constexpr (PST) {
        pst_solve_row<NB, REF>(d.P, d.F[sb], d.F[sb ^ 1], d.L[next_list(lb)], d.gstart, d.W, d.sc, i);
    } else {
        S.dt1 = d.dt1[S.stage - 1];
        S.dt2 = d.dt2[S.stage - 1];
        stage_solve_row<NB, REF>(d.P, d.F[sb], d.F[sb ^ 1], d.L[next_list(lb)], d.gstart, d.W, S, d.sc, i);
    }
}

// =======================================================================================
// Small kernels (static: this header is compiled into more than one translation unit)
// =======================================================================================
// Scatter the interior particles of the current positions (standalone update_cell).
// A periodic domain has no ghost particles.  In place of the ghost launch this kernel does
// that launch's other duties in the step: clear the scatter counters of the cell list the
// preceding stage consumed, reset the U_max slot after PST, and count the step.
static __global__ void k_housekeep(const Phys P, int* zero_cnt, int reset_umax, Scalars* sc) {
    pdl_wait();
    const bool stop = halted(sc);
    if (zero_cnt && !stop)
        for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < P.ncell; c += gridDim.x * blockDim.x) zero_cnt[c] = 0;
    if (reset_umax && blockIdx.x == 0 && threadIdx.x == 0) sc->umax2 = 0ull;
    pdl_release();
    if (reset_umax) end_of_step(sc, gridDim.x);
}

static __global__ void k_scatter(const Phys P, const Fld F, const Lst Ln, const int* __restrict__ gstart, int* key,
                          Scalars* sc) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.num_int) return;
    const int k = cell_key_mul(P, F.x[i], F.y[i], sc);
    if (k >= 0) key[i] = k;
    scatter_to_cell(P, Ln, gstart, k, i, sc);
}

static __global__ void k_umax(const Phys P, const Fld F, Scalars* sc) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double v = 0.0;
    if (i < P.num_int) v = F.u[i] * F.u[i] + F.v[i] * F.v[i];
    warp_max_atomic(&sc->umax2, v);
}

static __global__ void k_steady_max(const Phys P, const Fld F, const Work W, Scalars* sc) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double v = 0.0;
    if (i < P.num_int) v = fabs(W.f_prev[i] - F.u[i]);
    warp_max_atomic(&sc->dfmax, v);
}

static __global__ void k_copy_fprev(const Phys P, const Fld F, const Work W) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < P.num_int) W.f_prev[i] = F.u[i];
}

// Problem 1 epilogue of a step (main.f90:139-149 with check_steady_state_mod.f90:39-65):
// the stage kernel already reduced max|f_previous - u|.
// End of a time step of problem 1 (one thread): steady check, step count, step budget.
__device__ __forceinline__ void epilogue_body(double threshold, Scalars* sc) {
    pdl_wait();
    if (sc->err != 0 || sc->steady != 0 || sc->done != 0) return;
    sc->step_count += 1;
    const double df = __longlong_as_double((long long)sc->dfmax);
    if (df < threshold) {
        sc->steady = 1;
        sc->steady_step = sc->step_count;
    }
    if (sc->step_limit > 0 && sc->step_count >= sc->step_limit) sc->done = 1;
    sc->dfmax = 0ull;
}

static __global__ void k_epilogue(const Phys P, Scalars* sc) { epilogue_body(P.threshold, sc); }

// End of a batched step: advance the step counter the batched kernels read their buffer
// parities from (one graph then serves every step).
static __global__ void kb_advance(int* tstep) { *tstep = (*tstep + 1) % (2 * kLists); }

// Problem-1 epilogue for every solve of a batch (one thread per solve).
static __global__ void kb_epilogue(const SolveDesc* __restrict__ D, int nsolve) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < nsolve) epilogue_body(D[s].P.threshold, D[s].sc);
}

// Copy every batch member's scalars into one array (one read-back per batch call).
static __global__ void kb_gather_scalars(const SolveDesc* __restrict__ D, int nsolve, Scalars* out) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < nsolve) out[s] = *D[s].sc;
}

// Split-precision positions of every particle in both state buffers from the positions of
// A: interior particles by their cell keys, ghosts by the static cell that lists them.
static __global__ void k_split_pos(const Phys P, const Fld A, const Fld B, const int* __restrict__ key,
                                   const int* __restrict__ gstart, const int* __restrict__ glist) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < P.num_int) {
        const int k = key[t];
        if (k >= 0 && k < P.ncell) {
            put_split_pos(P, A, t, A.x[t], A.y[t], k);
            put_split_pos(P, B, t, A.x[t], A.y[t], k);
        }
    }
    if (t < P.ncell)
        for (int g = gstart[t]; g < gstart[t + 1]; ++g) {
            const int j = glist[g];
            put_split_pos(P, A, j, A.x[j], A.y[j], t);
            put_split_pos(P, B, j, A.x[j], A.y[j], t);
        }
}

static __global__ void k_volume(const Phys P, const Fld F) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < P.num_total) F.vol[i] = P.SP_mass / F.rho[i];
}

// Host state in page-locked, mapped memory (device addresses of the caller's buffers; a
// null field is left as it is on the device).
struct HostFld {
    const double *x, *y, *u, *v, *rho, *pre, *tem;
};
struct HostOut {
    double *x, *y, *u, *v, *rho, *pre, *tem;
};

// Upload read straight from mapped host memory (one pass over PCIe instead of one copy per
// field): every particle into the current buffer A, particles from `first_b` on into the
// other buffer B, and the volumes of both.
static __global__ void k_upload_mapped(const Phys P, const Fld A, const Fld B, const HostFld H, int first_b) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.num_total) return;
    const bool toB = i >= first_b;
    auto put = [&](const double* src, double* a, double* b) {
        if (!src) return;
        const double v = src[i];
        a[i] = v;
        if (toB) b[i] = v;
    };
    put(H.x, A.x, B.x);
    put(H.y, A.y, B.y);
    put(H.u, A.u, B.u);
    put(H.v, A.v, B.v);
    put(H.rho, A.rho, B.rho);
    put(H.pre, A.pre, B.pre);
    put(H.tem, A.tem, B.tem);
    A.vol[i] = P.SP_mass / A.rho[i];
    if (toB) B.vol[i] = P.SP_mass / B.rho[i];
}

// Download written straight into mapped host memory.
static __global__ void k_download_mapped(const Phys P, const Fld F, const HostOut H) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.num_total) return;
    if (H.x) H.x[i] = F.x[i];
    if (H.y) H.y[i] = F.y[i];
    if (H.u) H.u[i] = F.u[i];
    if (H.v) H.v[i] = F.v[i];
    if (H.rho) H.rho[i] = F.rho[i];
    if (H.pre) H.pre[i] = F.pre[i];
    if (H.tem) H.tem[i] = F.tem[i];
}

// Counters of the rotating cell lists to zero (one launch for all of them).
static __global__ void k_clear_counts(int* a, int* b, int* c, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) { a[i] = 0; b[i] = 0; c[i] = 0; }
}

// In-radius neighbour lists for parity checks (unsorted, fixed stride per particle).
static __global__ void k_neighbors(const Phys P, const Fld F, const Lst L, const int* __restrict__ gstart,
                            const int* __restrict__ glist, const int* key, const VMd V, int which, int stride,
                            int* out, int* count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = which == 0 ? P.num_int : P.num_ext;
    if (i >= n) return;
    const double mx = which == 0 ? F.x[i] : V.x[i];
    const double my = which == 0 ? F.y[i] : V.y[i];
    const int k = which == 0 ? key[i] : V.key[i];
    int c = 0;
    auto f = [&](int j, double sx, double sy) {
        if (which == 0 && j == i) return;
        const double xj = (F.x[j] + sx) - mx, yj = (F.y[j] + sy) - my;
        if (xj * xj + yj * yj > P.h_eff_sq) return;
        if (c < stride) out[(size_t)i * stride + c] = j;
        ++c;
    };
    if (which == 0) for_candidates<false>(P, L, gstart, glist, k, f);
    else for_candidates<true>(P, L, gstart, glist, k, f);
    count[i] = c;
}

}  // namespace lssph
