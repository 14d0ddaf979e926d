// kernels_hi.cuh -- higher-order LS-SPH (SPH_MODEL 4 / 5 / 6: Taylor order k = 3 / 4 / 5,
// q = 9 / 14 / 20 basis terms), FP64, sm_100a.
//
//   k_stage_hi   LSSPH_A (LSSPH_A_mod.f90:26-271) for k >= 3, fused with the RK stage
//                update, EOS and cell scatter exactly like k_stage
//   k_pst_hi     shift_interpolate (shift_interpolate_mod.f90:23-300) with the same q
//
// A q = 20 moment matrix (210 packed entries) and its b vectors (100 entries) do not fit
// in one thread's registers, so the work of a particle is spread over a whole warp:
//   1. the warp tests the particle's candidates 32 at a time and compacts the hits with a
//      ballot, which keeps the reference visiting order (cells, then list order);
//   2. for a chunk of up to 32 hits, lane t evaluates the pair terms of hit t (weight,
//      basis, field differences) into a per-warp shared-memory table;
//   3. each lane owns a fixed set of accumulator entries -- moment entries (i, j), b
//      entries (i, c) and, for PST, the two shift sums -- and adds every hit of the chunk
//      to them in order: entry (u, v) accumulates fma(U[h][u], V[h][v], .), where U holds
//      V_j W_ij a_i and V holds a_j and the differences.  That is the oracle's sequence for
//      each entry (the same fma chain over the same hit order), so the sums are
//      bit-identical to the oracle's for any lane count;
//   4. the entries go to a per-warp q x (q + nb) shared-memory matrix (symmetric fill),
//      lane i loads row i, and the warp runs the oracle's GEPP (first max |a| pivot,
//      reciprocal column scaling, right-looking update, then forward and back
//      substitution per right-hand side) with one matrix row per lane;
//   5. lane 0 gathers the solution and finishes the particle like the q = 5 kernels.
// Staging (the tile halo in shared memory) is shared with the q = 5 kernels.
#pragma once

#include "kernels.cuh"

namespace lssph {

// Number of basis terms for Taylor order k (LSSPH_A_mod.f90:46-56).
__host__ __device__ constexpr int q_of_order(int k) {
    return k == 1 ? 2 : k == 2 ? 5 : k == 3 ? 9 : k == 4 ? 14 : 20;
}

// Taylor basis of order K (LSSPH_A_mod.f90:140-172), the oracle's operation sequence.
template <int K>
__device__ __forceinline__ void basis_hi(double x, double y, const double (&ih)[5], double (&a)[q_of_order(K)]) {
    a[0] = x * ih[0];
    a[1] = y * ih[0];
    const double x2 = x * x, y2 = y * y;
    a[2] = (0.5 * x2) * ih[1];
    a[3] = (0.5 * y2) * ih[1];
    a[4] = (x * y) * ih[1];
    if constexpr (K >= 3) {
        const double x3 = x2 * x, y3 = y2 * y;
        a[5] = ((1.0 / 6.0) * x3) * ih[2];
        a[6] = ((1.0 / 6.0) * y3) * ih[2];
        a[7] = ((0.5 * x2) * y) * ih[2];
        a[8] = ((0.5 * y2) * x) * ih[2];
        if constexpr (K >= 4) {
            const double x4 = x2 * x2, y4 = y2 * y2;
            a[9] = ((1.0 / 24.0) * x4) * ih[3];
            a[10] = ((1.0 / 24.0) * y4) * ih[3];
            a[11] = (((1.0 / 6.0) * x3) * y) * ih[3];
            a[12] = (((1.0 / 6.0) * y3) * x) * ih[3];
            a[13] = (((1.0 / 4.0) * x2) * y2) * ih[3];
            if constexpr (K >= 5) {
                const double x5 = x4 * x, y5 = y4 * y;
                a[14] = ((1.0 / 120.0) * x5) * ih[4];
                a[15] = ((1.0 / 120.0) * y5) * ih[4];
                a[16] = (((1.0 / 24.0) * x4) * y) * ih[4];
                a[17] = (((1.0 / 24.0) * y4) * x) * ih[4];
                a[18] = (((1.0 / 12.0) * x3) * y2) * ih[4];
                a[19] = (((1.0 / 12.0) * y3) * x2) * ih[4];
            }
        }
    }
}

// Shapes of one warp-per-particle LS problem: Q basis terms, NBV right-hand sides, and
// (SHIFT) the two PST shift sums.  Pair table rows: U = [V_j W a_0..a_{Q-1} (, fac)],
// V = [a_0..a_{Q-1}, df_0..df_{NBV-1} (, gx, gy)].
template <int K, int NBV, bool SHIFT>
struct HiShape {
    static constexpr int Q = q_of_order(K);
    static constexpr int NBv = NBV;
    static constexpr bool kShift = SHIFT;
    static constexpr int QU = Q * (Q + 1) / 2;
    static constexpr int NU = Q + (SHIFT ? 1 : 0);
    static constexpr int NV = Q + NBV + (SHIFT ? 2 : 0);
    static constexpr int E = QU + Q * NBV + (SHIFT ? 2 : 0);   // accumulator entries
    static constexpr int PER = (E + 31) / 32;                   // entries per lane
    static constexpr int CH = 32;                               // hits per chunk
    static constexpr int US = NU | 1, VS = NV | 1;              // odd row strides (banks)
    static constexpr int MS = (Q + NBV) | 1;                    // matrix row stride
    static constexpr int TABLE = CH * (US + VS);                // doubles per warp
    static constexpr int MAT = Q * MS;
    static constexpr int WARP_DOUBLES = TABLE > MAT ? TABLE : MAT;
    static_assert(Q <= 32, "one matrix row per lane");
};

constexpr int HI_WARPS = 4;   // warps (particles in flight) per CTA

// Dynamic shared memory of a higher-order CTA: staged fields, lists, per-warp hit lists
// (which double as the staging scratch) and per-warp pair tables / matrices.
template <class S>
__host__ __device__ inline size_t hi_smem_bytes(int cap, bool tem) {
    const size_t maxp = (size_t)HC * cap, maxo = (size_t)OC * cap;
    const size_t hits = (size_t)HI_WARPS * 9 * cap;
    const size_t scratch = hits > maxp ? hits : maxp;
    return (size_t)HI_WARPS * S::WARP_DOUBLES * sizeof(double) + maxp * ((tem ? 8 : 7) * sizeof(double) + sizeof(int)) +
           2 * maxo * sizeof(int) + scratch * sizeof(int);
}

template <class S, bool TEM>
__device__ __forceinline__ SmemView hi_smem_view(void* raw, int cap, double*& warp_area) {
    SmemView V;
    const int maxp = HC * cap, maxo = OC * cap;
    double* d = static_cast<double*>(raw);
    warp_area = d;
    d += HI_WARPS * S::WARP_DOUBLES;
    V.sums = nullptr;
    V.x = d; V.y = d + maxp; V.u = d + 2 * maxp; V.v = d + 3 * maxp; V.rho = d + 4 * maxp;
    V.pre = d + 5 * maxp; V.vol = d + 6 * maxp; V.tem = TEM ? d + 7 * maxp : nullptr;
    int* q = reinterpret_cast<int*>(d + (TEM ? 8 : 7) * maxp);
    V.idx = q; V.own_k = q + maxp; V.own_hc = q + maxp + maxo;
    V.nbr = reinterpret_cast<unsigned short*>(q + maxp + 2 * maxo);
    return V;
}

// Hits of one particle, in the reference order, into `hits`; returns their number.
__device__ __forceinline__ int warp_hits(const TileHdr& T, const SmemView& SM, int hc, int self, double mx, double my,
                                         double h_eff_sq, int* hits) {
    const int lane = threadIdx.x & 31;
    int n = 0;
#pragma unroll 1
    for (int dy = -1; dy <= 1; ++dy) {
        const int lo = T.off[hc - 1 + dy * HX], hi = T.off[hc + 2 + dy * HX];
#pragma unroll 1
        for (int k0 = lo; k0 < hi; k0 += 32) {
            const int k = k0 + lane;
            bool hit = false;
            if (k < hi) {
                const double xji = SM.x[k] - mx;
                const double yji = SM.y[k] - my;
                hit = k != self && !(xji * xji + yji * yji > h_eff_sq);
            }
            const unsigned m = __ballot_sync(0xffffffffu, hit);
            if (hit) hits[n + __popc(m & ((1u << lane) - 1u))] = k;
            n += __popc(m);
        }
    }
    __syncwarp();
    return n;
}

// Entry e of a lane -> (u, v) column pair of the pair table; -1 past the last entry.
template <class S>
__device__ __forceinline__ void hi_entry(int e, int& u, int& v) {
    if (e < S::QU) {   // column-packed upper triangle, e = i (i + 1) / 2 + j, j <= i
        int i = 0;
        while ((i + 1) * (i + 2) / 2 <= e) ++i;
        u = i;
        v = e - i * (i + 1) / 2;
    } else if (e < S::QU + S::Q * S::NBv) {
        const int f = e - S::QU;   // b entry (i, c), e = QU + c Q + i
        u = f % S::Q;
        v = S::Q + f / S::Q;
    } else if (e < S::E) {         // shift sums: fac * gx, fac * gy
        u = S::Q;
        v = S::NV - 2 + (e - (S::E - 2));
    } else {
        u = -1;
        v = -1;
    }
}

// Steps 2-3 for all hits of a particle: `pair(h, k, urow, vrow)` writes the table rows of
// hit h (staged index k); acc[] gets this lane's entries.
template <class S, class Pair>
__device__ __forceinline__ void hi_accumulate(const int* hits, int n, double* wa, const int (&eu)[S::PER],
                                              const int (&ev)[S::PER], double (&acc)[S::PER], Pair&& pair) {
    const int lane = threadIdx.x & 31;
    double* U = wa;
    double* V = wa + S::CH * S::US;
#pragma unroll
    for (int t = 0; t < S::PER; ++t) acc[t] = 0.0;
#pragma unroll 1
    for (int c0 = 0; c0 < n; c0 += S::CH) {
        const int m = min(S::CH, n - c0);
        if (lane < m) pair(lane, hits[c0 + lane], U + lane * S::US, V + lane * S::VS);
        __syncwarp();
#pragma unroll 4
        for (int h = 0; h < m; ++h) {
            const double* u = U + h * S::US;
            const double* v = V + h * S::VS;
#pragma unroll
            for (int t = 0; t < S::PER; ++t)
                if (eu[t] >= 0) acc[t] = fma(u[eu[t]], v[ev[t]], acc[t]);
        }
        __syncwarp();
    }
}

// Step 4: entries -> symmetric matrix rows, lane i < Q loads row i (A) and its b entries
// (B), then the oracle's GEPP with one row per lane.  Returns false on a zero pivot
// (the same test as the oracle: the pivot column below the diagonal is all zero).
template <class S, int NB>
__device__ __forceinline__ bool hi_solve(double* wa, const int (&eu)[S::PER], const int (&ev)[S::PER],
                                         const double (&acc)[S::PER], double (&B)[NB]) {
    constexpr int Q = S::Q;
    const int lane = threadIdx.x & 31;
    double* Mx = wa;   // Q rows of stride MS: M(i, 0..Q-1), then b(i, 0..NB-1)
#pragma unroll
    for (int t = 0; t < S::PER; ++t) {
        const int u = eu[t], v = ev[t];
        if (u < 0) continue;
        if (v < Q) {               // moment entry (row v, col u), v <= u
            Mx[u * S::MS + v] = acc[t];
            Mx[v * S::MS + u] = acc[t];
        } else if (v < Q + NB) {   // b entry (i = u, c = v - Q)
            Mx[u * S::MS + v] = acc[t];
        }
    }
    __syncwarp();
    double A[Q];
    const int r = lane < Q ? lane : 0;
#pragma unroll
    for (int j = 0; j < Q; ++j) A[j] = Mx[r * S::MS + j];
#pragma unroll
    for (int c = 0; c < NB; ++c) B[c] = Mx[r * S::MS + Q + c];
    __syncwarp();
    const bool live = lane < Q;
    bool ok = true;
    double rpiv = 0.0;   // 1 / A(lane, lane) once this lane's row is the pivot row
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        // pivot: the oracle starts from row k and moves to a later row only when its
        // |A(i,k)| is strictly larger, i.e. the first row of the largest value; a NaN never
        // wins a comparison.  Max-reduction over the non-NaN rows >= k, ties to the
        // smaller row (associative, so every lane gets the same row).
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
        if (apk != 0.0 && p != k) {   // swap rows k and p (all columns and right-hand sides)
            const int src = lane == k ? p : (lane == p ? k : lane);
#pragma unroll
            for (int j = 0; j < Q; ++j) A[j] = __shfl_sync(0xffffffffu, A[j], src);
#pragma unroll
            for (int c = 0; c < NB; ++c) B[c] = __shfl_sync(0xffffffffu, B[c], src);
        }
        // after the interchange the diagonal is apk; the oracle's scaling reciprocal and
        // its stored reciprocal pivot are both 1 / A(k,k), one division serves both
        const double rk = 1.0 / apk;
        if (apk != 0.0) {
            if (lane > k) A[k] = A[k] * rk;
        } else {
            ok = false;
        }
        if (lane == k) rpiv = rk;
        // right-looking update of the trailing block: A(i,j) -= A(i,k) A(k,j)
#pragma unroll
        for (int j = k + 1; j < Q; ++j) {
            const double akj = __shfl_sync(0xffffffffu, A[j], k);
            if (lane > k) A[j] = fma(-A[k], akj, A[j]);
        }
    }
    // forward substitution (unit lower), then back substitution; each right-hand side
    // gets the oracle's sequence, the NB independent sequences are interleaved
#pragma unroll
    for (int k = 0; k < Q; ++k) {
#pragma unroll
        for (int c = 0; c < NB; ++c) {
            const double bk = __shfl_sync(0xffffffffu, B[c], k);
            if (lane > k) B[c] = fma(-bk, A[k], B[c]);
        }
    }
#pragma unroll
    for (int k = Q - 1; k >= 0; --k) {
#pragma unroll
        for (int c = 0; c < NB; ++c) {
            if (lane == k) B[c] = B[c] * rpiv;
            const double bk = __shfl_sync(0xffffffffu, B[c], k);
            if (lane < k) B[c] = fma(-bk, A[k], B[c]);
        }
    }
    return ok;
}

// Per-lane entry map, computed once per CTA.
template <class S>
__device__ __forceinline__ void hi_entries(int (&eu)[S::PER], int (&ev)[S::PER]) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int t = 0; t < S::PER; ++t) hi_entry<S>(lane + 32 * t, eu[t], ev[t]);
}

__device__ __forceinline__ void inv_h_powers(const Phys& P, double (&ih)[5]) {
    ih[0] = P.ih1;   // inv_h(1) = 1/h; inv_h(i) = inv_h(i-1)/h (LSSPH_A_mod.f90:90-93)
#pragma unroll
    for (int i = 1; i < 5; ++i) ih[i] = ih[i - 1] / P.h;
}

// ---- LSSPH_A, order K >= 3, fused stage -------------------------------------------------
template <int K, int NB>
__device__ __forceinline__ void stage_body_hi(const Phys& P, const Fld& cur, const Fld& nxt, const Lst& Lc,
                                              const Lst& Ln, const int* __restrict__ gstart,
                                              const int* __restrict__ glist, const Work& W, const StageCfg& Sc,
                                              Scalars* sc, int ntx, int tile) {
    using S = HiShape<K, NB, false>;
    constexpr int Q = S::Q;
    pdl_wait();
    const bool stop = halted(sc);
    __shared__ TileHdr T;
    extern __shared__ double smem_raw[];
    double* warp_area;
    const SmemView SM = hi_smem_view<S, NB == 5>(smem_raw, P.cap, warp_area);
    const int tx = tile % ntx, ty = tile / ntx;
    stage_halo<false, NB == 5>(P, cur, Lc, gstart, glist, tx * TX - 1, ty * TY - 1, T, SM);
    pdl_release();
    if (stop) return;
    const int n_own = T.own_off[OC];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double* wa = warp_area + warp * S::WARP_DOUBLES;
    int* hits = reinterpret_cast<int*>(SM.nbr) + warp * 9 * P.cap;
    int eu[S::PER], ev[S::PER];
    hi_entries<S>(eu, ev);
    double ih[5];
    inv_h_powers(P, ih);
    double red = 0.0;
#pragma unroll 1
    for (int o = warp; o < n_own; o += HI_WARPS) {
        const int ki = SM.own_k[o], hc = SM.own_hc[o];
        const double my_x = SM.x[ki], my_y = SM.y[ki], my_u = SM.u[ki];
        double my_v = 0, my_rho = 0, my_pre = 0, my_tem = 0;
        if constexpr (NB >= 4) { my_v = SM.v[ki]; my_rho = SM.rho[ki]; my_pre = SM.pre[ki]; }
        if constexpr (NB == 5) my_tem = SM.tem[ki];
        const int n = warp_hits(T, SM, hc, ki, my_x, my_y, P.h_eff_sq, hits);
        double acc[S::PER];
        hi_accumulate<S>(hits, n, wa, eu, ev, acc, [&](int, int k, double* u, double* v) {
            const double xji = SM.x[k] - my_x, yji = SM.y[k] - my_y;
            const double r = sqrt(xji * xji + yji * yji);
            const double Wv = dev_W<double>(P.kt, r, P.ih1, P.wnorm);
            const double VW = SM.vol[k] * Wv;
            double a[Q];
            basis_hi<K>(xji, yji, ih, a);
#pragma unroll
            for (int i = 0; i < Q; ++i) { u[i] = VW * a[i]; v[i] = a[i]; }
            v[Q] = SM.u[k] - my_u;
            if constexpr (NB >= 4) {
                v[Q + 1] = SM.v[k] - my_v;
                v[Q + 2] = SM.rho[k] - my_rho;
                v[Q + 3] = SM.pre[k] - my_pre;
            }
            if constexpr (NB == 5) v[Q + 4] = SM.tem[k] - my_tem;
        });
        double B[NB];
        if (n >= Q) {
            if (!hi_solve<S, NB>(wa, eu, ev, acc, B) && lane == 0) atomicOr(&sc->warn, WARN_SINGULAR);
        } else {
#pragma unroll
            for (int c = 0; c < NB; ++c) B[c] = 0.0;
        }
        // derivatives: entries 0..4 of each solution (x, y, xx, yy, xy)
        double d[NB][5];
#pragma unroll
        for (int c = 0; c < NB; ++c)
#pragma unroll
            for (int m = 0; m < 5; ++m) d[c][m] = __shfl_sync(0xffffffffu, B[c], m) * (m < 2 ? ih[0] : ih[1]);
        __syncwarp();
        if (lane == 0) {
            double Ru, Rv, Rr, Rt;
            rhs_ls<NB>(P, W, SM.idx[ki], my_rho, my_tem, d, Ru, Rv, Rr, Rt);
            red = fmax(red, stage_advance<NB>(P, nxt, Ln, gstart, W, Sc, sc, SM.idx[ki], my_x, my_y, my_u, my_v,
                                              my_rho, my_tem, Ru, Rv, Rr, Rt));
        }
    }
    if (Sc.mode == MODE_STAGE && Sc.last && (Sc.do_umax || Sc.do_steady))
        warp_max_atomic(Sc.do_umax ? &sc->umax2 : &sc->dfmax, red);
}

template <int K, int NB>
__global__ void __launch_bounds__(32 * HI_WARPS)
    k_stage_hi(const Phys P, const Fld cur, const Fld nxt, const Lst Lc, const Lst Ln, const int* __restrict__ gstart,
               const int* __restrict__ glist, const Work W, const StageCfg S, Scalars* sc, int ntx,
               const int* __restrict__ tiles) {
    stage_body_hi<K, NB>(P, cur, nxt, Lc, Ln, gstart, glist, W, S, sc, ntx, tiles ? tiles[blockIdx.x] : (int)blockIdx.x);
}

// ---- shift_interpolate, order K >= 3, fused PST -----------------------------------------
// NB = 3 (u, v, rho) or 4 (+T).
template <int K, int NB>
__device__ __forceinline__ void pst_body_hi(const Phys& P, const Fld& cur, const Fld& nxt, const Lst& Lc,
                                            const Lst& Ln, const int* __restrict__ gstart,
                                            const int* __restrict__ glist, const Work& W, Scalars* sc, int ntx,
                                            int tile) {
    using S = HiShape<K, NB, true>;
    constexpr int Q = S::Q;
    pdl_wait();
    const bool stop = halted(sc);
    __shared__ TileHdr T;
    extern __shared__ double smem_raw[];
    double* warp_area;
    const SmemView SM = hi_smem_view<S, NB == 4>(smem_raw, P.cap, warp_area);
    const int tx = tile % ntx, ty = tile / ntx;
    stage_halo<false, NB == 4>(P, cur, Lc, gstart, glist, tx * TX - 1, ty * TY - 1, T, SM);
    pdl_release();
    if (stop) return;
    const int n_own = T.own_off[OC];
    const double U_max = sqrt(__longlong_as_double((long long)sc->umax2));
    const double coe = ((P.PST_c * U_max) * P.dt) * P.h;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double* wa = warp_area + warp * S::WARP_DOUBLES;
    int* hits = reinterpret_cast<int*>(SM.nbr) + warp * 9 * P.cap;
    int eu[S::PER], ev[S::PER];
    hi_entries<S>(eu, ev);
    double ih[5];
    inv_h_powers(P, ih);
#pragma unroll 1
    for (int o = warp; o < n_own; o += HI_WARPS) {
        const int ki = SM.own_k[o], hc = SM.own_hc[o];
        const double my_x = SM.x[ki], my_y = SM.y[ki], my_u = SM.u[ki], my_v = SM.v[ki], my_rho = SM.rho[ki];
        double my_tem = 0.0;
        if constexpr (NB == 4) my_tem = SM.tem[ki];
        const int n = warp_hits(T, SM, hc, ki, my_x, my_y, P.h_eff_sq, hits);
        double acc[S::PER];
        hi_accumulate<S>(hits, n, wa, eu, ev, acc, [&](int, int k, double* u, double* v) {
            const double xji = SM.x[k] - my_x, yji = SM.y[k] - my_y;
            const double r = sqrt(xji * xji + yji * yji);
            const double Wv = dev_W<double>(P.kt, r, P.ih1, P.wnorm);
            const double dWdr = dev_dW<double>(P.kt, r, P.ih1, P.m3h, P.m5h, P.wnorm);
            const double Vj = SM.vol[k];
            const double VW = Vj * Wv;
            const double rinv = 1.0 / r;
            const double t = Wv * P.iWave, t2 = t * t, t4 = t2 * t2;
            double a[Q];
            basis_hi<K>(xji, yji, ih, a);
#pragma unroll
            for (int i = 0; i < Q; ++i) { u[i] = VW * a[i]; v[i] = a[i]; }
            u[Q] = 1.0 + 0.2 * t4;
            v[Q] = SM.u[k] - my_u;
            v[Q + 1] = SM.v[k] - my_v;
            v[Q + 2] = SM.rho[k] - my_rho;
            if constexpr (NB == 4) v[Q + 3] = SM.tem[k] - my_tem;
            v[Q + NB] = ((dWdr * (-xji)) * rinv) * Vj;
            v[Q + NB + 1] = ((dWdr * (-yji)) * rinv) * Vj;
        });
        // the shift sums are the last two entries
        double sx = 0.0, sy = 0.0;
#pragma unroll
        for (int t = 0; t < S::PER; ++t) {
            if (lane + 32 * t == S::E - 2) sx = acc[t];
            if (lane + 32 * t == S::E - 1) sy = acc[t];
        }
        sx = __shfl_sync(0xffffffffu, sx, (S::E - 2) & 31);
        sy = __shfl_sync(0xffffffffu, sy, (S::E - 1) & 31);
        double B[NB];
        if (n >= Q) {
            if (!hi_solve<S, NB>(wa, eu, ev, acc, B) && lane == 0) atomicOr(&sc->warn, WARN_SINGULAR);
        } else {
#pragma unroll
            for (int c = 0; c < NB; ++c) B[c] = 0.0;
        }
        // shift vector, clamped to 0.2 h (shift_interpolate_mod.f90:216-225)
        double dx = -coe * sx, dy = -coe * sy;
        const double rr = sqrt(dx * dx + dy * dy);
        if (rr > 0.2 * P.h) {
            dx = ((0.2 * P.h) * dx) / rr;
            dy = ((0.2 * P.h) * dy) / rr;
        }
        // interpolation a(dr) . d (shift_interpolate_mod.f90:255-298), terms in order
        double a[Q];
        basis_hi<K>(dx, dy, ih, a);
        double accf[NB];
#pragma unroll
        for (int c = 0; c < NB; ++c) {
            double s = 0.0;
#pragma unroll
            for (int i = 0; i < Q; ++i) s = fma(a[i], __shfl_sync(0xffffffffu, B[c], i), s);
            accf[c] = s;
        }
        __syncwarp();
        if (lane == 0) {
            const int i = SM.idx[ki];
            double xn = my_x + dx, yn = my_y + dy;
            if (P.periodic) { xn = wrap_pos(xn, P.Lx); yn = wrap_pos(yn, P.Lx); }
            const double un = my_u + accf[0], vn = my_v + accf[1], rn = my_rho + accf[2];
            nxt.x[i] = xn; nxt.y[i] = yn; nxt.u[i] = un; nxt.v[i] = vn; nxt.rho[i] = rn;
            nxt.pre[i] = P.c_sq * (rn - P.rho_ref);
            nxt.vol[i] = P.SP_mass / rn;
            bool finite = isfinite(xn) && isfinite(yn) && isfinite(un) && isfinite(vn) && isfinite(rn);
            if constexpr (NB == 4) { const double tn = my_tem + accf[3]; nxt.tem[i] = tn; finite = finite && isfinite(tn); }
            if (!finite) atomicOr(&sc->err, ERR_NONFINITE);
            const int nk = cell_key_mul(P, xn, yn, sc);
            if (nk >= 0) W.key[i] = nk;
            scatter_to_cell(P, Ln, gstart, nk, i, sc);
        }
    }
}

template <int K, int NB>
__global__ void __launch_bounds__(32 * HI_WARPS)
    k_pst_hi(const Phys P, const Fld cur, const Fld nxt, const Lst Lc, const Lst Ln, const int* __restrict__ gstart,
             const int* __restrict__ glist, const Work W, Scalars* sc, int ntx, const int* __restrict__ tiles) {
    pst_body_hi<K, NB>(P, cur, nxt, Lc, Ln, gstart, glist, W, sc, ntx, tiles ? tiles[blockIdx.x] : (int)blockIdx.x);
}


// =======================================================================================
// Thread-per-particle variant.  Each thread owns one particle and a private slot of shared
// memory holding its moment matrix, right-hand sides and reciprocal pivots (element e of
// thread t at slot[e * NT + t], so a warp's accesses to one element are conflict-free).
// The thread runs the oracle's loops verbatim -- accumulation over its hits in reference
// order, symmetric fill, GEPP, substitutions -- so results are again bit-identical, and a
// warp advances 32 particles per instruction instead of one.  Hits are found in chunks of
// HCH per thread (16-bit staged indices), so a particle with many neighbours resumes its
// candidate scan where the previous chunk stopped.
// =======================================================================================
template <int K, int NBV, bool SHIFT>
struct TppShape {
    static constexpr int Q = q_of_order(K);
    static constexpr int NB = NBV;
    // threads (particles in flight) per CTA: a tile has about 24 particles, and every thread
    // holds a Q x Q slot, so 32 (not 64) threads leave room for twice the CTAs per SM
    // (q = 9 on B200: 28-44% faster at 128^2-256^2)
    static constexpr int NT = 32;
    static constexpr int SLOT = Q * Q + Q * NBV + Q;   // A (row-major), B (column-major), 1/pivots
    static constexpr int HCH = 32;                     // hits per chunk
    static constexpr int EA = 0, EB = Q * Q, ER = Q * Q + Q * NBV;
};

template <class S>
__host__ __device__ inline size_t tpp_smem_bytes(int cap, bool tem) {
    const size_t maxp = (size_t)HC * cap, maxo = (size_t)OC * cap;
    const size_t hl = (size_t)S::NT * S::HCH * 2;
    const size_t scratch = maxp * sizeof(int) > hl ? maxp * sizeof(int) : hl;
    return (size_t)S::NT * S::SLOT * sizeof(double) + maxp * ((tem ? 8 : 7) * sizeof(double) + sizeof(int)) +
           2 * maxo * sizeof(int) + scratch;
}

template <class S, bool TEM>
__device__ __forceinline__ SmemView tpp_smem_view(void* raw, int cap, double*& slots) {
    SmemView V;
    const int maxp = HC * cap, maxo = OC * cap;
    double* d = static_cast<double*>(raw);
    slots = d;
    d += S::NT * S::SLOT;
    V.sums = nullptr;
    V.x = d; V.y = d + maxp; V.u = d + 2 * maxp; V.v = d + 3 * maxp; V.rho = d + 4 * maxp;
    V.pre = d + 5 * maxp; V.vol = d + 6 * maxp; V.tem = TEM ? d + 7 * maxp : nullptr;
    int* q = reinterpret_cast<int*>(d + (TEM ? 8 : 7) * maxp);
    V.idx = q; V.own_k = q + maxp; V.own_hc = q + maxp + maxo;
    V.nbr = reinterpret_cast<unsigned short*>(q + maxp + 2 * maxo);   // staging scratch, then the per-thread hit chunks
    return V;
}

// Visit this thread's hits (reference order) in chunks; f(k) per hit.  Returns the count.
template <class S, class F>
__device__ __forceinline__ int tpp_pairs(const TileHdr& T, const SmemView& SM, int hc, int self, double mx, double my,
                                         double h_eff_sq, F&& f) {
    unsigned short* hl = reinterpret_cast<unsigned short*>(SM.nbr) + threadIdx.x;
    int row = 0, k = T.off[hc - 1 - HX], total = 0;
    bool more = true;
    while (more) {
        int nh = 0;
        while (row < 3 && nh < S::HCH) {
            const int hi = T.off[hc + 2 + (row - 1) * HX];
            for (; k < hi && nh < S::HCH; ++k) {
                const double xji = SM.x[k] - mx;
                const double yji = SM.y[k] - my;
                if (k != self && !(xji * xji + yji * yji > h_eff_sq)) hl[(nh++) * S::NT] = (unsigned short)k;
            }
            if (k >= hi) {
                ++row;
                if (row < 3) k = T.off[hc - 1 + (row - 1) * HX];
            }
        }
        more = row < 3;
#pragma unroll 1
        for (int t = 0; t < nh; ++t) f((int)hl[t * S::NT]);
        total += nh;
    }
    return total;
}

#define TA(r, c) sl[(S::EA + (r) * S::Q + (c)) * S::NT]
#define TB(r, c) sl[(S::EB + (c) * S::Q + (r)) * S::NT]
#define TR(k) sl[(S::ER + (k)) * S::NT]

// The oracle's GEPP + substitutions on one thread's slot (sl[e * NT] = element e).
// Returns false on a zero pivot.
template <class S>
__device__ __forceinline__ bool tpp_solve(double* sl) {
    constexpr int Q = S::Q, NB = S::NB;
    // elimination steps are unrolled for q = 9 only: unrolled q = 14 / 20 code would not
    // fit the instruction cache
    constexpr int UK = Q <= 9 ? Q : 1;
    bool ok = true;
#pragma unroll UK
    for (int k = 0; k < Q; ++k) {
        int p = k;
        double amax = fabs(TA(k, k));
#pragma unroll
        for (int i = k + 1; i < Q; ++i) {
            const double a = fabs(TA(i, k));
            if (a > amax) { amax = a; p = i; }
        }
        const double apk = TA(p, k);
        if (apk != 0.0 && p != k) {
#pragma unroll
            for (int c = 0; c < Q; ++c) { const double t = TA(k, c); TA(k, c) = TA(p, c); TA(p, c) = t; }
#pragma unroll
            for (int c = 0; c < NB; ++c) { const double t = TB(k, c); TB(k, c) = TB(p, c); TB(p, c) = t; }
        }
        // the scaling reciprocal and the stored reciprocal pivot are both 1 / A(k,k)
        const double rk = 1.0 / apk;
        if (apk != 0.0) {
#pragma unroll
            for (int i = k + 1; i < Q; ++i) TA(i, k) = TA(i, k) * rk;
        } else {
            ok = false;
        }
        TR(k) = rk;
#pragma unroll
        for (int j = k + 1; j < Q; ++j) {
            const double akj = TA(k, j);
#pragma unroll
            for (int i = k + 1; i < Q; ++i) TA(i, j) = fma(-TA(i, k), akj, TA(i, j));
        }
    }
#pragma unroll UK
    for (int k = 0; k < Q; ++k) {
        double bk[NB];
#pragma unroll
        for (int c = 0; c < NB; ++c) bk[c] = TB(k, c);
#pragma unroll
        for (int i = k + 1; i < Q; ++i) {
            const double aik = TA(i, k);
#pragma unroll
            for (int c = 0; c < NB; ++c) TB(i, c) = fma(-bk[c], aik, TB(i, c));
        }
    }
#pragma unroll UK
    for (int k = Q - 1; k >= 0; --k) {
        const double rp = TR(k);
        double bk[NB];
#pragma unroll
        for (int c = 0; c < NB; ++c) { bk[c] = TB(k, c) * rp; TB(k, c) = bk[c]; }
#pragma unroll
        for (int i = 0; i < k; ++i) {
            const double aik = TA(i, k);
#pragma unroll
            for (int c = 0; c < NB; ++c) TB(i, c) = fma(-bk[c], aik, TB(i, c));
        }
    }
    return ok;
}

// Zero A and B of a slot.
template <class S>
__device__ __forceinline__ void tpp_clear(double* sl) {
#pragma unroll
    for (int e = 0; e < S::ER; ++e) sl[e * S::NT] = 0.0;
}

// Lower triangle of A from its upper triangle (LSSPH_A_mod.f90:203-205).
template <class S>
__device__ __forceinline__ void tpp_symmetrize(double* sl) {
#pragma unroll
    for (int i = 1; i < S::Q; ++i)
#pragma unroll
        for (int j = 0; j < i; ++j) TA(i, j) = TA(j, i);
}

// One hit's contribution (LSSPH_A_mod.f90:174-188 / shift_interpolate_mod.f90:188-201):
// b(i, c) += V W a_i df_c, M(j, i) += V W a_i a_j for j <= i.
template <class S>
__device__ __forceinline__ void tpp_accumulate(double* sl, double VW, const double (&a)[S::Q], const double (&df)[S::NB]) {
#pragma unroll
    for (int i = 0; i < S::Q; ++i) {
        const double VWa = VW * a[i];
#pragma unroll
        for (int c = 0; c < S::NB; ++c) TB(i, c) = fma(VWa, df[c], TB(i, c));
#pragma unroll
        for (int j = 0; j <= i; ++j) TA(j, i) = fma(VWa, a[j], TA(j, i));
    }
}

template <int K, int NB>
__device__ __forceinline__ void stage_body_tpp(const Phys& P, const Fld& cur, const Fld& nxt, const Lst& Lc,
                                               const Lst& Ln, const int* __restrict__ gstart,
                                               const int* __restrict__ glist, const Work& W, const StageCfg& Sc,
                                               Scalars* sc, int ntx, int tile) {
    using S = TppShape<K, NB, false>;
    constexpr int Q = S::Q;
    pdl_wait();
    const bool stop = halted(sc);
    __shared__ TileHdr T;
    extern __shared__ double smem_raw[];
    double* slots;
    const SmemView SM = tpp_smem_view<S, NB == 5>(smem_raw, P.cap, slots);
    const int tx = tile % ntx, ty = tile / ntx;
    stage_halo<false, NB == 5>(P, cur, Lc, gstart, glist, tx * TX - 1, ty * TY - 1, T, SM);
    pdl_release();
    if (stop) return;
    const int n_own = T.own_off[OC];
    double* sl = slots + threadIdx.x;
    double ih[5];
    inv_h_powers(P, ih);
    double red = 0.0;
#pragma unroll 1
    for (int o = threadIdx.x; o < n_own; o += S::NT) {
        const int ki = SM.own_k[o], hc = SM.own_hc[o];
        const double my_x = SM.x[ki], my_y = SM.y[ki], my_u = SM.u[ki];
        double my_v = 0, my_rho = 0, my_pre = 0, my_tem = 0;
        if constexpr (NB >= 4) { my_v = SM.v[ki]; my_rho = SM.rho[ki]; my_pre = SM.pre[ki]; }
        if constexpr (NB == 5) my_tem = SM.tem[ki];
        tpp_clear<S>(sl);
        const int n = tpp_pairs<S>(T, SM, hc, ki, my_x, my_y, P.h_eff_sq, [&](int k) {
            const double xji = SM.x[k] - my_x, yji = SM.y[k] - my_y;
            const double r = sqrt(xji * xji + yji * yji);
            const double Wv = dev_W<double>(P.kt, r, P.ih1, P.wnorm);
            const double VW = SM.vol[k] * Wv;
            double a[Q];
            basis_hi<K>(xji, yji, ih, a);
            double df[NB];
            df[0] = SM.u[k] - my_u;
            if constexpr (NB >= 4) {
                df[1] = SM.v[k] - my_v;
                df[2] = SM.rho[k] - my_rho;
                df[3] = SM.pre[k] - my_pre;
            }
            if constexpr (NB == 5) df[4] = SM.tem[k] - my_tem;
            tpp_accumulate<S>(sl, VW, a, df);
        });
        double d[NB][5];
        if (n >= Q) {
            tpp_symmetrize<S>(sl);
            if (!tpp_solve<S>(sl)) atomicOr(&sc->warn, WARN_SINGULAR);
#pragma unroll
            for (int c = 0; c < NB; ++c)
#pragma unroll
                for (int m = 0; m < 5; ++m) d[c][m] = TB(m, c) * (m < 2 ? ih[0] : ih[1]);
        } else {
#pragma unroll
            for (int c = 0; c < NB; ++c)
#pragma unroll
                for (int m = 0; m < 5; ++m) d[c][m] = 0.0;
        }
        const int i = SM.idx[ki];
        double Ru, Rv, Rr, Rt;
        rhs_ls<NB>(P, W, i, my_rho, my_tem, d, Ru, Rv, Rr, Rt);
        red = fmax(red, stage_advance<NB>(P, nxt, Ln, gstart, W, Sc, sc, i, my_x, my_y, my_u, my_v, my_rho, my_tem,
                                          Ru, Rv, Rr, Rt));
    }
    if (Sc.mode == MODE_STAGE && Sc.last && (Sc.do_umax || Sc.do_steady))
        warp_max_atomic(Sc.do_umax ? &sc->umax2 : &sc->dfmax, red);
}

template <int K, int NB>
__global__ void __launch_bounds__(TppShape<K, NB, false>::NT)
    k_stage_tpp(const Phys P, const Fld cur, const Fld nxt, const Lst Lc, const Lst Ln, const int* __restrict__ gstart,
                const int* __restrict__ glist, const Work W, const StageCfg S, Scalars* sc, int ntx,
                const int* __restrict__ tiles) {
    stage_body_tpp<K, NB>(P, cur, nxt, Lc, Ln, gstart, glist, W, S, sc, ntx, tiles ? tiles[blockIdx.x] : (int)blockIdx.x);
}

template <int K, int NB>
__device__ __forceinline__ void pst_body_tpp(const Phys& P, const Fld& cur, const Fld& nxt, const Lst& Lc,
                                             const Lst& Ln, const int* __restrict__ gstart,
                                             const int* __restrict__ glist, const Work& W, Scalars* sc, int ntx,
                                             int tile) {
    using S = TppShape<K, NB, true>;
    constexpr int Q = S::Q;
    pdl_wait();
    const bool stop = halted(sc);
    __shared__ TileHdr T;
    extern __shared__ double smem_raw[];
    double* slots;
    const SmemView SM = tpp_smem_view<S, NB == 4>(smem_raw, P.cap, slots);
    const int tx = tile % ntx, ty = tile / ntx;
    stage_halo<false, NB == 4>(P, cur, Lc, gstart, glist, tx * TX - 1, ty * TY - 1, T, SM);
    pdl_release();
    if (stop) return;
    const int n_own = T.own_off[OC];
    const double U_max = sqrt(__longlong_as_double((long long)sc->umax2));
    const double coe = ((P.PST_c * U_max) * P.dt) * P.h;
    double* sl = slots + threadIdx.x;
    double ih[5];
    inv_h_powers(P, ih);
#pragma unroll 1
    for (int o = threadIdx.x; o < n_own; o += S::NT) {
        const int ki = SM.own_k[o], hc = SM.own_hc[o];
        const double my_x = SM.x[ki], my_y = SM.y[ki], my_u = SM.u[ki], my_v = SM.v[ki], my_rho = SM.rho[ki];
        double my_tem = 0.0;
        if constexpr (NB == 4) my_tem = SM.tem[ki];
        tpp_clear<S>(sl);
        double sx = 0.0, sy = 0.0;
        const int n = tpp_pairs<S>(T, SM, hc, ki, my_x, my_y, P.h_eff_sq, [&](int k) {
            const double xji = SM.x[k] - my_x, yji = SM.y[k] - my_y;
            const double r = sqrt(xji * xji + yji * yji);
            const double Wv = dev_W<double>(P.kt, r, P.ih1, P.wnorm);
            const double dWdr = dev_dW<double>(P.kt, r, P.ih1, P.m3h, P.m5h, P.wnorm);
            const double Vj = SM.vol[k];
            const double VW = Vj * Wv;
            const double rinv = 1.0 / r;
            const double gx = ((dWdr * (-xji)) * rinv) * Vj;
            const double gy = ((dWdr * (-yji)) * rinv) * Vj;
            const double t = Wv * P.iWave, t2 = t * t, t4 = t2 * t2;
            const double fac = 1.0 + 0.2 * t4;
            sx = fma(fac, gx, sx);
            sy = fma(fac, gy, sy);
            double a[Q];
            basis_hi<K>(xji, yji, ih, a);
            double df[NB];
            df[0] = SM.u[k] - my_u;
            df[1] = SM.v[k] - my_v;
            df[2] = SM.rho[k] - my_rho;
            if constexpr (NB == 4) df[3] = SM.tem[k] - my_tem;
            tpp_accumulate<S>(sl, VW, a, df);
        });
        // shift vector, clamped to 0.2 h (shift_interpolate_mod.f90:216-225)
        double dx = -coe * sx, dy = -coe * sy;
        const double rr = sqrt(dx * dx + dy * dy);
        if (rr > 0.2 * P.h) {
            dx = ((0.2 * P.h) * dx) / rr;
            dy = ((0.2 * P.h) * dy) / rr;
        }
        double accf[NB];
        if (n >= Q) {
            tpp_symmetrize<S>(sl);
            if (!tpp_solve<S>(sl)) atomicOr(&sc->warn, WARN_SINGULAR);
            double a[Q];
            basis_hi<K>(dx, dy, ih, a);
#pragma unroll
            for (int c = 0; c < NB; ++c) {
                double s = 0.0;
#pragma unroll
                for (int i = 0; i < Q; ++i) s = fma(a[i], TB(i, c), s);
                accf[c] = s;
            }
        } else {
#pragma unroll
            for (int c = 0; c < NB; ++c) accf[c] = 0.0;
        }
        const int i = SM.idx[ki];
        double xn = my_x + dx, yn = my_y + dy;
        if (P.periodic) { xn = wrap_pos(xn, P.Lx); yn = wrap_pos(yn, P.Lx); }
        const double un = my_u + accf[0], vn = my_v + accf[1], rn = my_rho + accf[2];
        nxt.x[i] = xn; nxt.y[i] = yn; nxt.u[i] = un; nxt.v[i] = vn; nxt.rho[i] = rn;
        nxt.pre[i] = P.c_sq * (rn - P.rho_ref);
        nxt.vol[i] = P.SP_mass / rn;
        bool finite = isfinite(xn) && isfinite(yn) && isfinite(un) && isfinite(vn) && isfinite(rn);
        if constexpr (NB == 4) { const double tn = my_tem + accf[3]; nxt.tem[i] = tn; finite = finite && isfinite(tn); }
        if (!finite) atomicOr(&sc->err, ERR_NONFINITE);
        const int nk = cell_key_mul(P, xn, yn, sc);
        if (nk >= 0) W.key[i] = nk;
        scatter_to_cell(P, Ln, gstart, nk, i, sc);
    }
}
#undef TA
#undef TB
#undef TR

template <int K, int NB>
__global__ void __launch_bounds__(TppShape<K, NB, true>::NT)
    k_pst_tpp(const Phys P, const Fld cur, const Fld nxt, const Lst Lc, const Lst Ln, const int* __restrict__ gstart,
              const int* __restrict__ glist, const Work W, Scalars* sc, int ntx, const int* __restrict__ tiles) {
    pst_body_tpp<K, NB>(P, cur, nxt, Lc, Ln, gstart, glist, W, sc, ntx, tiles ? tiles[blockIdx.x] : (int)blockIdx.x);
}

}  // namespace lssph
