// postproc.cu -- LS type-B interpolation of one particle field at arbitrary points, the
// reference's post-processing step (analysis/common/lssph_b.py:21-143): the value and the two
// first derivatives at each point from every particle within h_eff, by the normal equations
// M = A^T W A, b = A^T W f with W = diag(W_ij V_j) and a pivoted elimination.  The
// reference runs a Python loop over the points with a KD-tree ball query and small numpy
// solves; its analysis scripts call it for the cavity and Taylor-Green velocity profiles,
// the Taylor-Green centre pressure and the wall Nusselt numbers.
//
// Device work of one call:
//   1. bin the particles into cells of width h_eff (count, exclusive scan, atomic fill, and a
//      rank sort per cell, so each cell lists its particles in ascending index and every
//      point's sums run in a fixed order);
//   2. one thread per point scans its 3 x 3 cells, accumulates M (packed upper triangle)
//      and b, and solves.  Fewer than q neighbours, or a zero pivot, gives NaN, as the
//      reference does (its numpy solve raises LinAlgError on an exactly singular matrix).
// q (3, 6, 10, 15, 21) follows SPH_MODEL and TARGET_PROBLEM as in lssph_b.py:45-55, with the
// reference's basis column orders.

#include <cuda_runtime.h>
#include <math_constants.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <string>

#include "handle.h"

namespace lssph {
namespace {

struct PGrid {
    double x0, y0, he;   // origin of cell (0,0) and the cell width h_eff
    int ncx, ncy;
};

struct PConst {
    double h, he2, ih1, wnorm, mass;
    int kt;
};

int post_q(int sph_model, int target_problem) {   // lssph_b.py:45-55
    const bool t4 = target_problem == 4;
    if (sph_model <= 3) return t4 ? 6 : 3;
    if (sph_model == 4) return t4 ? 10 : 6;
    if (sph_model == 5) return t4 ? 15 : 10;
    return t4 ? 21 : 15;
}

__device__ __forceinline__ int pp_cell(const PGrid& g, double x, double y) {
    const double fx = floor((x - g.x0) / g.he), fy = floor((y - g.y0) / g.he);
    const int cx = fx < 0.0 ? 0 : (fx > g.ncx - 1 ? g.ncx - 1 : (int)fx);
    const int cy = fy < 0.0 ? 0 : (fy > g.ncy - 1 ? g.ncy - 1 : (int)fy);
    return cx + cy * g.ncx;
}

__global__ void k_pp_bin(int n, const double* __restrict__ x, const double* __restrict__ y, double shift, PGrid g,
                         int* __restrict__ key, int* __restrict__ cnt) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const int c = pp_cell(g, x[j] - shift, y[j] - shift);
    key[j] = c;
    atomicAdd(cnt + c, 1);
}

// Exclusive scan of cnt[0..m) into start[0..m] (start[m] = total); one CTA of 1024 threads,
// each summing a contiguous run.
__global__ void __launch_bounds__(1024) k_pp_scan(int m, const int* __restrict__ cnt, int* __restrict__ start) {
    __shared__ int part[1024];
    const int t = threadIdx.x, per = (m + 1023) / 1024;
    const int b0 = min(m, t * per), b1 = min(m, b0 + per);
    int s = 0;
    for (int i = b0; i < b1; ++i) s += cnt[i];
    part[t] = s;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
        const int v = t >= off ? part[t - off] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    int run = t ? part[t - 1] : 0;
    for (int i = b0; i < b1; ++i) {
        start[i] = run;
        run += cnt[i];
    }
    if (t == 1023) start[m] = part[1023];
}

// Fill: each particle takes a slot of its cell by an atomic counter (arbitrary order) ...
__global__ void k_pp_fill(int n, const int* __restrict__ key, const int* __restrict__ start, int* __restrict__ cursor,
                          int* __restrict__ tmp) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const int c = key[j];
    tmp[start[c] + atomicAdd(cursor + c, 1)] = j;
}

// ... then one warp per cell puts its indices in ascending order (each index's rank is the
// number of smaller ones in the cell), so every point's sums run in a fixed order.
__global__ void k_pp_rank(int m, const int* __restrict__ start, const int* __restrict__ tmp, int* __restrict__ list) {
    const int c = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (c >= m) return;
    const int s0 = start[c], nc = start[c + 1] - s0;
    for (int i = lane; i < nc; i += 32) {
        const int v = tmp[s0 + i];
        int r = 0;
        for (int k = 0; k < nc; ++k) r += tmp[s0 + k] < v ? 1 : 0;
        list[s0 + r] = v;
    }
}

// Basis columns of lssph_b.py:83-125 on normalised offsets X = dx / h, Y = dy / h.
template <int Q>
__device__ __forceinline__ void pp_basis(double X, double Y, double (&a)[Q]) {
    a[0] = 1.0;
    a[1] = X;
    a[2] = Y;
    if constexpr (Q == 6 || Q == 10) {
        const double X2 = X * X, Y2 = Y * Y;
        a[3] = 0.5 * X2;
        a[4] = X * Y;
        a[5] = 0.5 * Y2;
        if constexpr (Q == 10) {
            a[6] = (1.0 / 6.0) * (X2 * X);
            a[7] = (0.5 * X2) * Y;
            a[8] = (0.5 * X) * Y2;
            a[9] = (1.0 / 6.0) * (Y2 * Y);
        }
    } else if constexpr (Q >= 15) {
        const double X2 = X * X, Y2 = Y * Y, X3 = X2 * X, Y3 = Y2 * Y, X4 = X2 * X2, Y4 = Y2 * Y2;
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
        if constexpr (Q == 21) {
            a[15] = (1.0 / 120.0) * (X4 * X);
            a[16] = (1.0 / 120.0) * (Y4 * Y);
            a[17] = ((1.0 / 24.0) * X4) * Y;
            a[18] = ((1.0 / 24.0) * Y4) * X;
            a[19] = ((1.0 / 12.0) * X3) * Y2;
            a[20] = ((1.0 / 12.0) * Y3) * X2;
        }
    }
}

// One thread per point.  Loops are unrolled (registers) for q <= 10; q = 15 / 21 keep
// the matrix in local memory.
template <int Q>
__global__ void __launch_bounds__(128) k_pp_points(PConst pc, PGrid g, double shift, const double* __restrict__ x,
                                                   const double* __restrict__ y, const double* __restrict__ val,
                                                   const double* __restrict__ rho, const int* __restrict__ start,
                                                   const int* __restrict__ list, int nt, const double* __restrict__ tx,
                                                   const double* __restrict__ ty, double* __restrict__ out) {
    constexpr int U = Q <= 10 ? Q : 1;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    const double px = tx[t], py = ty[t];
    double M[Q * (Q + 1) / 2], b[Q];
#pragma unroll
    for (int e = 0; e < Q * (Q + 1) / 2; ++e) M[e] = 0.0;
#pragma unroll
    for (int i = 0; i < Q; ++i) b[i] = 0.0;
    int n = 0;
    const double fx = floor((px - g.x0) / g.he), fy = floor((py - g.y0) / g.he);
    if (fx >= -1.0 && fx <= (double)g.ncx && fy >= -1.0 && fy <= (double)g.ncy) {
        const int cx = (int)fx, cy = (int)fy;
        for (int yy = max(cy - 1, 0); yy <= min(cy + 1, g.ncy - 1); ++yy)
            for (int xx = max(cx - 1, 0); xx <= min(cx + 1, g.ncx - 1); ++xx) {
                const int c = xx + yy * g.ncx;
                for (int s = start[c]; s < start[c + 1]; ++s) {
                    const int j = list[s];
                    const double dx = (x[j] - shift) - px, dy = (y[j] - shift) - py;
                    const double r2 = dx * dx + dy * dy;
                    if (r2 > pc.he2) continue;
                    ++n;
                    const double w = dev_W<double>(pc.kt, sqrt(r2), pc.ih1, pc.wnorm) * (pc.mass / rho[j]);
                    double a[Q];
                    pp_basis<Q>(dx / pc.h, dy / pc.h, a);
                    const double f = val[j];
#pragma unroll U
                    for (int i = 0; i < Q; ++i) {
                        const double wa = w * a[i];
                        b[i] = fma(wa, f, b[i]);
#pragma unroll U
                        for (int k = 0; k <= i; ++k) M[UT(k, i)] = fma(wa, a[k], M[UT(k, i)]);
                    }
                }
            }
    }
    double* o = out + 3 * (size_t)t;
    if (n < Q) {
        o[0] = o[1] = o[2] = CUDART_NAN;
        return;
    }
    // pivoted elimination on the full symmetric matrix (first largest |a| pivot)
    double A[Q][Q];
#pragma unroll U
    for (int r = 0; r < Q; ++r)
#pragma unroll U
        for (int c = 0; c < Q; ++c) A[r][c] = r <= c ? M[UT(r, c)] : M[UT(c, r)];
    bool ok = true;
#pragma unroll U
    for (int k = 0; k < Q; ++k) {
        int p = k;
        double amax = fabs(A[k][k]);
        for (int i = k + 1; i < Q; ++i)
            if (fabs(A[i][k]) > amax) { amax = fabs(A[i][k]); p = i; }
        if (A[p][k] == 0.0) { ok = false; break; }
        if (p != k) {
            for (int c = 0; c < Q; ++c) { const double s = A[k][c]; A[k][c] = A[p][c]; A[p][c] = s; }
            const double s = b[k]; b[k] = b[p]; b[p] = s;
        }
        const double rp = 1.0 / A[k][k];
        for (int i = k + 1; i < Q; ++i) {
            const double l = A[i][k] * rp;
            for (int c = k + 1; c < Q; ++c) A[i][c] = fma(-l, A[k][c], A[i][c]);
            b[i] = fma(-l, b[k], b[i]);
        }
    }
    if (!ok) {
        o[0] = o[1] = o[2] = CUDART_NAN;
        return;
    }
    for (int k = Q - 1; k >= 0; --k) {
        double s = b[k];
        for (int c = k + 1; c < Q; ++c) s = fma(-A[k][c], b[c], s);
        b[k] = s / A[k][k];
    }
    o[0] = b[0];
    o[1] = b[1] / pc.h;
    o[2] = b[2] / pc.h;
}

// ---- q >= 10: one warp per point ----------------------------------------------------------
// A q = 21 system (231 packed moments) does not fit one thread.  The warp compacts the hits
// with a ballot (same order as the thread kernel: cells row by row, ascending index within a
// cell), evaluates up to 32 hits at a time into a shared-memory table (w a_i, a_i, f), and
// each lane adds the table rows to its own accumulator entries in hit order -- the thread
// kernel's fma chain for each entry.  The pivoted elimination then runs with one matrix row
// per lane.
constexpr int PP_WARPS = 4;

template <int Q>
struct PPWarp {
    static constexpr int QU = Q * (Q + 1) / 2;
    static constexpr int E = QU + Q;              // moment entries, then b entries
    static constexpr int PER = (E + 31) / 32;
    static constexpr int RS = (2 * Q + 1) | 1;    // table row: w a_0..w a_{Q-1}, a_0..a_{Q-1}, f
    static constexpr int TABLE = 32 * RS;
    static constexpr int MS = (Q + 1) | 1;        // matrix row: M(i, 0..Q-1), b_i
    static constexpr int MAT = Q * MS;
    static constexpr int DOUBLES = TABLE > MAT ? TABLE : MAT;
    static constexpr size_t BYTES = (size_t)PP_WARPS * (DOUBLES * sizeof(double) + 64 * sizeof(int));
};

template <int Q>
__global__ void __launch_bounds__(32 * PP_WARPS) k_pp_points_warp(PConst pc, PGrid g, double shift,
                                                                 const double* __restrict__ x, const double* __restrict__ y,
                                                                 const double* __restrict__ val,
                                                                 const double* __restrict__ rho,
                                                                 const int* __restrict__ start,
                                                                 const int* __restrict__ list, int nt,
                                                                 const double* __restrict__ tx,
                                                                 const double* __restrict__ ty, double* __restrict__ out) {
    using S = PPWarp<Q>;
    extern __shared__ double pp_smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int t = blockIdx.x * PP_WARPS + warp;
    if (t >= nt) return;   // whole warp
    double* tab = pp_smem + warp * S::DOUBLES;
    int* hits = reinterpret_cast<int*>(pp_smem + PP_WARPS * S::DOUBLES) + warp * 64;
    // this lane's entries: e < QU -> moment (row j, col i), j <= i; else b_i
    int eu[S::PER], ev[S::PER];
#pragma unroll
    for (int k = 0; k < S::PER; ++k) {
        const int e = lane + 32 * k;
        if (e < S::QU) {
            int i = 0;
            while ((i + 1) * (i + 2) / 2 <= e) ++i;
            eu[k] = i;
            ev[k] = Q + (e - i * (i + 1) / 2);   // a_j in the table's second block
        } else if (e < S::E) {
            eu[k] = e - S::QU;
            ev[k] = 2 * Q;                        // f
        } else {
            eu[k] = -1;
            ev[k] = 0;
        }
    }
    double acc[S::PER];
#pragma unroll
    for (int k = 0; k < S::PER; ++k) acc[k] = 0.0;
    const double px = tx[t], py = ty[t];
    int n = 0, pending = 0;
    // evaluate hits[0..m) into the table, add them to the entries
    auto flush = [&](int m) {
        if (lane < m) {
            const int j = hits[lane];
            const double dx = (x[j] - shift) - px, dy = (y[j] - shift) - py;
            const double w = dev_W<double>(pc.kt, sqrt(dx * dx + dy * dy), pc.ih1, pc.wnorm) * (pc.mass / rho[j]);
            double a[Q];
            pp_basis<Q>(dx / pc.h, dy / pc.h, a);
            double* row = tab + lane * S::RS;
#pragma unroll
            for (int i = 0; i < Q; ++i) { row[i] = w * a[i]; row[Q + i] = a[i]; }
            row[2 * Q] = val[j];
        }
        __syncwarp();
#pragma unroll 1
        for (int h = 0; h < m; ++h) {
            const double* row = tab + h * S::RS;
#pragma unroll
            for (int k = 0; k < S::PER; ++k)
                if (eu[k] >= 0) acc[k] = fma(row[eu[k]], row[ev[k]], acc[k]);
        }
        __syncwarp();
    };
    const double fx = floor((px - g.x0) / g.he), fy = floor((py - g.y0) / g.he);
    if (fx >= -1.0 && fx <= (double)g.ncx && fy >= -1.0 && fy <= (double)g.ncy) {
        const int cx = (int)fx, cy = (int)fy;
        for (int yy = max(cy - 1, 0); yy <= min(cy + 1, g.ncy - 1); ++yy)
            for (int xx = max(cx - 1, 0); xx <= min(cx + 1, g.ncx - 1); ++xx) {
                const int c = xx + yy * g.ncx, s0 = start[c], s1 = start[c + 1];
                for (int b = s0; b < s1; b += 32) {
                    const int s = b + lane;
                    bool hit = false;
                    int j = 0;
                    if (s < s1) {
                        j = list[s];
                        const double dx = (x[j] - shift) - px, dy = (y[j] - shift) - py;
                        hit = !(dx * dx + dy * dy > pc.he2);
                    }
                    const unsigned mk = __ballot_sync(0xffffffffu, hit);
                    if (hit) hits[pending + __popc(mk & ((1u << lane) - 1u))] = j;
                    pending += __popc(mk);
                    n += __popc(mk);
                    __syncwarp();
                    if (pending >= 32) {   // evaluate 32, keep the rest (< 32) at the front
                        flush(32);
                        if (lane < pending - 32) hits[lane] = hits[32 + lane];
                        pending -= 32;
                        __syncwarp();
                    }
                }
            }
    }
    if (pending > 0) flush(pending);
    double* o = out + 3 * (size_t)t;
    if (n < Q) {
        if (lane == 0) o[0] = o[1] = o[2] = CUDART_NAN;
        return;
    }
    // symmetric matrix rows; lane r < Q loads row r (M(r, 0..Q-1), b_r)
    double* Mx = tab;
#pragma unroll
    for (int k = 0; k < S::PER; ++k) {
        if (eu[k] < 0) continue;
        if (ev[k] < 2 * Q) {
            const int i = eu[k], j = ev[k] - Q;
            Mx[i * S::MS + j] = acc[k];
            Mx[j * S::MS + i] = acc[k];
        } else {
            Mx[eu[k] * S::MS + Q] = acc[k];
        }
    }
    __syncwarp();
    const bool live = lane < Q;
    const int r = live ? lane : 0;
    double A[Q];
#pragma unroll
    for (int j = 0; j < Q; ++j) A[j] = Mx[r * S::MS + j];
    double bv = Mx[r * S::MS + Q];
    bool ok = true;
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        // pivot: the first row >= k with the largest |A(i,k)|; NaN never wins
        const double mine = fabs(A[k]);
        const double akk = __shfl_sync(0xffffffffu, mine, k);
        double av = (live && lane >= k && !isnan(mine)) ? mine : -1.0;
        int ai = lane;
#pragma unroll
        for (int off = 16; off >= 1; off >>= 1) {
            const double ov = __shfl_xor_sync(0xffffffffu, av, off);
            const int oi = __shfl_xor_sync(0xffffffffu, ai, off);
            if (ov > av || (ov == av && oi < ai)) { av = ov; ai = oi; }
        }
        const int p = (isnan(akk) || !(av > akk)) ? k : ai;
        const double apk = __shfl_sync(0xffffffffu, A[k], p);
        if (apk == 0.0) { ok = false; break; }
        if (p != k) {
            const int src = lane == k ? p : (lane == p ? k : lane);
#pragma unroll
            for (int j = 0; j < Q; ++j) A[j] = __shfl_sync(0xffffffffu, A[j], src);
            bv = __shfl_sync(0xffffffffu, bv, src);
        }
        const double l = A[k] * (1.0 / apk);
#pragma unroll
        for (int j = k + 1; j < Q; ++j) {
            const double akj = __shfl_sync(0xffffffffu, A[j], k);
            if (lane > k) A[j] = fma(-l, akj, A[j]);
        }
        const double bk = __shfl_sync(0xffffffffu, bv, k);
        if (lane > k) bv = fma(-l, bk, bv);
    }
    if (!ok) {
        if (lane == 0) o[0] = o[1] = o[2] = CUDART_NAN;
        return;
    }
    // back substitution, column by column
#pragma unroll
    for (int k = Q - 1; k >= 0; --k) {
        if (lane == k) bv = bv / A[k];
        const double bk = __shfl_sync(0xffffffffu, bv, k);
        if (lane < k) bv = fma(-A[k], bk, bv);
    }
    const double d0 = __shfl_sync(0xffffffffu, bv, 0), d1 = __shfl_sync(0xffffffffu, bv, 1),
                 d2 = __shfl_sync(0xffffffffu, bv, 2);
    if (lane == 0) {
        o[0] = d0;
        o[1] = d1 / pc.h;
        o[2] = d2 / pc.h;
    }
}

template <int Q>
void launch_points(const PConst& pc, const PGrid& g, double shift, const double* x, const double* y,
                   const double* val, const double* rho, const int* start, const int* list, int nt, const double* tx,
                   const double* ty, double* out, cudaStream_t st) {
    if constexpr (Q >= 10) {
        k_pp_points_warp<Q><<<(nt + PP_WARPS - 1) / PP_WARPS, 32 * PP_WARPS, PPWarp<Q>::BYTES, st>>>(
            pc, g, shift, x, y, val, rho, start, list, nt, tx, ty, out);
    } else {
        k_pp_points<Q><<<(nt + 127) / 128, 128, 0, st>>>(pc, g, shift, x, y, val, rho, start, list, nt, tx, ty, out);
    }
}

// Scratch of one call, carved from one stream-ordered allocation.
struct PBufs {
    void* block = nullptr;
    double *x = nullptr, *y = nullptr, *val = nullptr, *rho = nullptr, *tx = nullptr, *ty = nullptr, *out = nullptr;
    int *key = nullptr, *cnt = nullptr, *start = nullptr, *cursor = nullptr, *list = nullptr;
};

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

// Bin particles (device pointers x, y), interpolate `val` at the device points, write
// 3 * nt doubles to dout.  All work on stream st.
cudaError_t interpolate_device(const lssph_params& p, int n, const double* x, const double* y, const double* val,
                               const double* rho, double shift, const PGrid& g, int nt, const double* tx,
                               const double* ty, double* dout, int* key, int* cnt, int* start, int* cursor, int* tmp,
                               int* list, cudaStream_t st, const char** stage) {
    const int m = g.ncx * g.ncy;
    *stage = "clearing the bin counters";
    cudaError_t e = cudaMemsetAsync(cnt, 0, sizeof(int) * (size_t)m, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(cursor, 0, sizeof(int) * (size_t)m, st);
    if (e != cudaSuccess) return e;
    *stage = "k_pp_bin";
    if (n > 0) k_pp_bin<<<(n + 255) / 256, 256, 0, st>>>(n, x, y, shift, g, key, cnt);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    *stage = "k_pp_scan";
    k_pp_scan<<<1, 1024, 0, st>>>(m, cnt, start);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    *stage = "k_pp_fill";
    if (n > 0) {
        k_pp_fill<<<(n + 255) / 256, 256, 0, st>>>(n, key, start, cursor, tmp);
        k_pp_rank<<<(m + 3) / 4, 128, 0, st>>>(m, start, tmp, list);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    *stage = "k_pp_points";
    PConst pc;
    pc.h = p.h;
    pc.he2 = p.h_eff * p.h_eff;
    pc.ih1 = 1.0 / p.h;
    pc.wnorm = kernel_norm(p.kernel_type, p.h);
    pc.mass = p.SP_mass;
    pc.kt = p.kernel_type;
    if (nt > 0) {
        switch (post_q(p.sph_model, p.target_problem)) {
            case 3: launch_points<3>(pc, g, shift, x, y, val, rho, start, list, nt, tx, ty, dout, st); break;
            case 6: launch_points<6>(pc, g, shift, x, y, val, rho, start, list, nt, tx, ty, dout, st); break;
            case 10: launch_points<10>(pc, g, shift, x, y, val, rho, start, list, nt, tx, ty, dout, st); break;
            case 15: launch_points<15>(pc, g, shift, x, y, val, rho, start, list, nt, tx, ty, dout, st); break;
            default: launch_points<21>(pc, g, shift, x, y, val, rho, start, list, nt, tx, ty, dout, st); break;
        }
    }
    return cudaGetLastError();
}

// Cell grid over [lo, hi] with width h_eff, at most 2^24 cells.
bool make_grid(double x0, double y0, double x1, double y1, double he, PGrid* g) {
    if (!(he > 0.0) || !std::isfinite(x0) || !std::isfinite(x1) || !std::isfinite(y0) || !std::isfinite(y1))
        return false;
    const double nx = std::floor((x1 - x0) / he) + 1.0, ny = std::floor((y1 - y0) / he) + 1.0;
    if (nx * ny > (double)(1 << 24)) return false;
    g->x0 = x0;
    g->y0 = y0;
    g->he = he;
    g->ncx = (int)nx;
    g->ncy = (int)ny;
    return true;
}

int pp_fail(lssph_handle* h, int code, const std::string& msg) {
    if (h) h->err = msg;
    set_last_error(msg);
    return code;
}

}  // namespace
}  // namespace lssph

namespace lssph {

// A call's private stream, its event and a grow-only device scratch, kept between calls:
// creating a stream and drawing a few MB from the stream-ordered pool (which hands the
// memory back at every synchronisation) cost about 0.55 ms per call, several times the
// interpolation itself.
struct PPScratch {
    cudaStream_t st = nullptr;
    cudaEvent_t ev = nullptr;
    char* buf = nullptr;
    size_t bytes = 0;
};

// Stream and event on first use; a scratch of at least `bytes` (a larger one replaces it).
cudaError_t pp_ready(PPScratch* s, size_t bytes, const char** stage) {
    cudaError_t e = cudaSuccess;
    *stage = "stream set-up";
    if (!s->st) e = cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking);
    if (e == cudaSuccess && !s->ev) e = cudaEventCreateWithFlags(&s->ev, cudaEventDisableTiming);
    if (e == cudaSuccess && s->bytes < bytes) {
        *stage = "cudaMalloc of the scratch";
        if (s->buf) cudaFree(s->buf);
        s->buf = nullptr;
        s->bytes = 0;
        e = cudaMalloc((void**)&s->buf, bytes);
        if (e == cudaSuccess) s->bytes = bytes;
    }
    return e;
}

void pp_free(PPScratch* s) {
    if (!s) return;
    if (s->st) cudaStreamSynchronize(s->st);
    if (s->buf) cudaFree(s->buf);
    if (s->ev) cudaEventDestroy(s->ev);
    if (s->st) cudaStreamDestroy(s->st);
    delete s;
}

void postproc_release(lssph_handle* h) {
    pp_free(h->pp);
    h->pp = nullptr;
}

namespace {
// lssph_lsb_interpolate has no handle: one scratch per device, one call at a time per
// device, kept until the process exits.
std::mutex g_pp_mu[64];
PPScratch g_pp[64];
}  // namespace

}  // namespace lssph

using namespace lssph;

extern "C" {

int lssph_lsb_interpolate(const lssph_params* p, int32_t n, const double* x, const double* y, const double* val,
                          const double* rho, int32_t n_targets, const double* tx, const double* ty, double* out) {
    if (!p || n < 0 || n_targets < 0 || (n > 0 && (!x || !y || !val || !rho)) ||
        (n_targets > 0 && (!tx || !ty || !out)))
        return pp_fail(nullptr, LSSPH_E_BAD_PARAM, "lssph_lsb_interpolate: bad argument");
    if (!(p->h > 0.0) || !(p->h_eff > 0.0) || p->kernel_type < 1 || p->kernel_type > 5)
        return pp_fail(nullptr, LSSPH_E_BAD_PARAM, "lssph_lsb_interpolate: h, h_eff and kernel_type must be set");
    if (n_targets == 0) return LSSPH_OK;
    cudaGetLastError();   // a pending error of an unrelated earlier call is not this call's
    PGrid g{0.0, 0.0, p->h_eff, 1, 1};
    if (n > 0) {
        double x0 = x[0], x1 = x[0], y0 = y[0], y1 = y[0];
        for (int j = 1; j < n; ++j) {
            x0 = std::min(x0, x[j]); x1 = std::max(x1, x[j]);
            y0 = std::min(y0, y[j]); y1 = std::max(y1, y[j]);
        }
        if (!make_grid(x0, y0, x1, y1, p->h_eff, &g))
            return pp_fail(nullptr, LSSPH_E_BAD_PARAM,
                           "lssph_lsb_interpolate: particle positions must be finite and span at most 2^24 cells");
    }
    const size_t N = (size_t)std::max(n, 1), T = (size_t)n_targets, C = (size_t)g.ncx * g.ncy;
    const size_t bytes = 4 * align256(8 * N) + 2 * align256(8 * T) + align256(8 * 3 * T) + 3 * align256(4 * N) +
                         3 * align256(4 * (C + 1));
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
        return pp_fail(nullptr, LSSPH_E_CUDA, "lssph_lsb_interpolate: no usable CUDA device");
    std::lock_guard<std::mutex> lock(g_pp_mu[dev]);
    PPScratch& S = g_pp[dev];
    const char* stage = "";
    cudaError_t e = pp_ready(&S, bytes, &stage);
    cudaStream_t st = S.st;
    char* blk = S.buf;
    if (e == cudaSuccess) {
        size_t off = 0;
        auto carve = [&](size_t b) { char* q = blk + off; off += align256(b); return q; };
        double* dx = (double*)carve(8 * N);
        double* dy = (double*)carve(8 * N);
        double* dv = (double*)carve(8 * N);
        double* dr = (double*)carve(8 * N);
        double* dtx = (double*)carve(8 * T);
        double* dty = (double*)carve(8 * T);
        double* dout = (double*)carve(8 * 3 * T);
        int* key = (int*)carve(4 * N);
        int* list = (int*)carve(4 * N);
        int* tmp = (int*)carve(4 * N);
        int* cnt = (int*)carve(4 * (C + 1));
        int* start = (int*)carve(4 * (C + 1));
        int* cursor = (int*)carve(4 * (C + 1));
        if (off > bytes)   // the carve must stay inside the allocation
            return pp_fail(nullptr, LSSPH_E_CUDA, "lssph_lsb_interpolate: scratch layout exceeds its allocation");
        if (n > 0) {
            cudaMemcpyAsync(dx, x, 8 * (size_t)n, cudaMemcpyHostToDevice, st);
            cudaMemcpyAsync(dy, y, 8 * (size_t)n, cudaMemcpyHostToDevice, st);
            cudaMemcpyAsync(dv, val, 8 * (size_t)n, cudaMemcpyHostToDevice, st);
            cudaMemcpyAsync(dr, rho, 8 * (size_t)n, cudaMemcpyHostToDevice, st);
        }
        cudaMemcpyAsync(dtx, tx, 8 * T, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(dty, ty, 8 * T, cudaMemcpyHostToDevice, st);
        e = interpolate_device(*p, n, dx, dy, dv, dr, 0.0, g, n_targets, dtx, dty, dout, key, cnt, start, cursor,
                               tmp, list, st, &stage);
        if (e == cudaSuccess) {
            stage = "copy of the results";
            e = cudaMemcpyAsync(out, dout, 8 * 3 * T, cudaMemcpyDeviceToHost, st);
        }
        const cudaError_t e2 = cudaStreamSynchronize(st);
        if (e == cudaSuccess && e2 != cudaSuccess) {
            stage = "stream synchronize";
            e = e2;
        }
    }
    if (e != cudaSuccess)
        return pp_fail(nullptr, LSSPH_E_CUDA,
                       std::string("lssph_lsb_interpolate: ") + stage + ": " + cudaGetErrorString(e));
    return LSSPH_OK;
}

int lssph_interpolate(lssph_handle* h, int32_t field, int32_t n_targets, const double* tx, const double* ty,
                      double* out) {
    if (!h) return pp_fail(nullptr, LSSPH_E_BAD_PARAM, "null handle");
    if (n_targets < 0 || (n_targets > 0 && (!tx || !ty || !out)))
        return pp_fail(h, LSSPH_E_BAD_PARAM, "lssph_interpolate: bad argument");
    const Fld& F = h->F[h->sb];
    const double* val = field == LSSPH_FIELD_U ? F.u : field == LSSPH_FIELD_V ? F.v : field == LSSPH_FIELD_RHO ? F.rho
                        : field == LSSPH_FIELD_PRE ? F.pre : (field == LSSPH_FIELD_TEM && h->has_tem) ? F.tem : nullptr;
    if (!val) return pp_fail(h, LSSPH_E_BAD_PARAM, "lssph_interpolate: unknown field (or temperature without problem 4)");
    if (n_targets == 0) return LSSPH_OK;
    cudaGetLastError();   // a pending error of an unrelated earlier call is not this call's
    // particle positions in the physical frame (x - WL_thick), as the analysis scripts use;
    // they stay inside the solver's cell grid, so that grid's extent bounds the bins
    const double wl = h->p.WL_thick;
    PGrid g{-wl, -wl, h->p.h_eff, h->grid.nx, h->grid.ny};
    const size_t N = (size_t)h->num_total, T = (size_t)n_targets, C = (size_t)g.ncx * g.ncy;
    const size_t bytes = 2 * align256(8 * T) + align256(8 * 3 * T) + 3 * align256(4 * N) + 3 * align256(4 * (C + 1));
    // the handle's private stream, started after the handle's queued work
    if (!h->pp) h->pp = new PPScratch();
    const char* stage = "";
    cudaError_t e = pp_ready(h->pp, bytes, &stage);
    cudaStream_t st = h->pp->st;
    char* blk = h->pp->buf;
    if (e == cudaSuccess) e = cudaEventRecord(h->pp->ev, h->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(st, h->pp->ev, 0);
    if (e == cudaSuccess) {
        size_t off = 0;
        auto carve = [&](size_t b) { char* q = blk + off; off += align256(b); return q; };
        double* dtx = (double*)carve(8 * T);
        double* dty = (double*)carve(8 * T);
        double* dout = (double*)carve(8 * 3 * T);
        int* key = (int*)carve(4 * N);
        int* list = (int*)carve(4 * N);
        int* tmp = (int*)carve(4 * N);
        int* cnt = (int*)carve(4 * (C + 1));
        int* start = (int*)carve(4 * (C + 1));
        int* cursor = (int*)carve(4 * (C + 1));
        stage = "copy of the points";
        if (off > bytes) {   // the carve must stay inside the allocation
            stage = "scratch layout";
            e = cudaErrorInvalidValue;
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(dtx, tx, 8 * T, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(dty, ty, 8 * T, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) {
            e = interpolate_device(h->p, h->num_total, F.x, F.y, val, F.rho, wl, g, n_targets, dtx, dty, dout, key,
                                   cnt, start, cursor, tmp, list, st, &stage);
        }
        if (e == cudaSuccess) {
            stage = "copy of the results";
            e = cudaMemcpyAsync(out, dout, 8 * 3 * T, cudaMemcpyDeviceToHost, st);
        }
        const cudaError_t e2 = cudaStreamSynchronize(st);
        if (e == cudaSuccess && e2 != cudaSuccess) {
            stage = "stream synchronize";
            e = e2;
        }
    }
    if (e != cudaSuccess)
        return pp_fail(h, LSSPH_E_CUDA, std::string("lssph_interpolate: ") + stage + ": " + cudaGetErrorString(e));
    return LSSPH_OK;
}

}  // extern "C"
