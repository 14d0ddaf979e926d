// engine.cu -- device-resident LS-SPH solve: memory layout, launch sequences, graph
// replay of the time loop, and the handle half of the C ABI (lssph.h).
//
// HBM layout of one solve (all SoA, FP64 unless noted):
//   state      2 buffers x {x, y, u, v, rho, pre, tem, vol} over num_total (ping-pong:
//              a stage reads one buffer and writes the other, so neighbour gathers never
//              see half-updated particles); vol = SP_mass / rho is kept beside rho
//   work       x/y/u/v/rho/tem _old and _acc (RK4 accumulators), RHS arrays, f_previous,
//              the problem-1 source term, int32 cell key, over num_int
//   cell list  2 buffers x {cnt over ncell, slots[ncell * cap]} (int32), interior
//              particles in scatter order; static ghost lists per cell (CSR)
//   markers    virtual-marker positions, normals, keys and interpolated values, plus
//              the static list of cell tiles that hold markers
// Kernels work on tiles of 2 x 2 cells staged in shared memory.  A time step of
// problems 2-4 is 10 kernels (4 x {stage, ghost} + {pst, ghost}); problem 1 is 5
// (2 x {stage, ghost} + epilogue).  Each step is captured once in a CUDA graph and
// replayed.

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "engine.h"
#include "handle.h"
#include "hostmem.h"

using namespace lssph;


namespace {

// Page-locked slots for the handles' scalar read-back, shared by the process: page-locking
// a buffer per handle (and unlocking it at destroy) cost about 2 ms per handle, half of a
// handle's create + destroy.  Chunks of slots are locked on demand and kept; a handle takes
// a slot at create and returns it at destroy, after its stream has drained.  Portable, so
// that handles on any device of the process can use a slot.
std::mutex g_pin_mu;
std::vector<Scalars*> g_pin_free;
constexpr int kPinChunk = 256;

Scalars* pinned_slot() {
    std::lock_guard<std::mutex> lock(g_pin_mu);
    if (g_pin_free.empty()) {
        Scalars* chunk = nullptr;
        if (cudaHostAlloc((void**)&chunk, sizeof(Scalars) * kPinChunk, cudaHostAllocPortable) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;   // the checks then copy through pageable memory
        }
        for (int k = kPinChunk - 1; k >= 0; --k) g_pin_free.push_back(chunk + k);
    }
    Scalars* s = g_pin_free.back();
    g_pin_free.pop_back();
    return s;
}

void return_pinned_slot(Scalars* s) {
    if (!s) return;
    std::lock_guard<std::mutex> lock(g_pin_mu);
    g_pin_free.push_back(s);
}

int fail(lssph_handle* h, int code, const std::string& msg) {
    if (h) h->err = msg;
    set_last_error(msg);
    return code;
}

#define CUDA_TRY(h, call)                                                                      \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
            return fail((h), LSSPH_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// Every device array of a solve, in one place: the visitor gets (&pointer, element count)
// for each.  Used to size the solve's single device block and to carve it up.
template <class Vis>
void visit_solve_arrays(lssph_handle* h, size_t N, size_t NI, size_t NE, size_t NC, int cap, int nvt, int ntiles,
                        Vis&& A) {
    for (int b = 0; b < 2; ++b) {
        Fld& F = h->F[b];
        A(&F.x, N); A(&F.y, N); A(&F.u, N); A(&F.v, N); A(&F.rho, N); A(&F.pre, N); A(&F.tem, N); A(&F.vol, N);
        A(&F.ox, N); A(&F.oy, N);
    }
    for (int b = 0; b < kLists; ++b) {
        Lst& L = h->L[b];
        A(&L.cnt, NC); A(&L.slots, NC * (size_t)cap);
    }
    Work& W = h->W;
    A(&W.x_old, NI); A(&W.y_old, NI); A(&W.u_old, NI); A(&W.v_old, NI); A(&W.rho_old, NI); A(&W.tem_old, NI);
    A(&W.x_acc, NI); A(&W.y_acc, NI); A(&W.u_acc, NI); A(&W.v_acc, NI); A(&W.rho_acc, NI); A(&W.tem_acc, NI);
    A(&W.rhs_u, NI); A(&W.rhs_v, NI); A(&W.rhs_rho, NI); A(&W.rhs_tem, NI);
    A(&W.f_prev, NI); A(&W.src, NI); A(&W.key, NI);
    A(&W.sums, h->has_sums ? NI * MXS_ENTRIES : 0);   // the split shape's pair sums
    VMd& V = h->V;
    A(&V.x, NE); A(&V.y, NE); A(&V.nx, NE); A(&V.ny, NE); A(&V.u, NE); A(&V.v, NE); A(&V.pre, NE); A(&V.tem, NE);
    A(&V.K, NE); A(&V.ptype, NE); A(&V.key, NE); A(&V.mode, NE);
    A(&h->gstart, NC + 1); A(&h->glist, NE);
    A(&h->sc, 1);
    A(&h->vt_tile, (size_t)std::max(nvt, 1)); A(&h->vt_start, (size_t)nvt + 1); A(&h->vt_vm, NE);
    A(&h->tile_int, (size_t)ntiles); A(&h->tile_wall, (size_t)ntiles);
}

constexpr size_t kArrayAlign = 256;   // every array starts on a 256-byte boundary
inline size_t align_up(size_t v) { return (v + kArrayAlign - 1) / kArrayAlign * kArrayAlign; }

template <class T>
size_t array_bytes(T**, size_t n) { return align_up(std::max<size_t>(n, 1) * sizeof(T)); }

// Virtual markers grouped by the cell tile that holds them, in chunks of at most PPB
// markers (one pass of a ghost CTA): chunk tile ids, chunk ranges, marker ids.
void vm_chunks(const CellGrid& g, int ntx, int ntiles, std::vector<int32_t>* tile, std::vector<int32_t>* start,
               std::vector<int32_t>* vm) {
    const size_t NE = g.vm_key.size();
    std::vector<std::vector<int32_t>> by_tile(ntiles);
    for (size_t me = 0; me < NE; ++me) {
        const int key = g.vm_key[me];
        const int cx = key % g.nx, cy = key / g.nx;
        by_tile[(cx / TX) + (cy / TY) * ntx].push_back((int32_t)me);
    }
    tile->clear();
    start->assign(1, 0);
    vm->assign(NE, 0);
    size_t k = 0;
    for (int t = 0; t < ntiles; ++t) {
        for (size_t b = 0; b < by_tile[t].size(); b += PPB) {
            tile->push_back(t);
            for (size_t e = b; e < std::min(by_tile[t].size(), b + PPB); ++e) (*vm)[k++] = by_tile[t][e];
            start->push_back((int32_t)k);
        }
    }
}

// Size of the single device block of a solve of these sizes (every array holds at least
// one element and starts on a 256-byte boundary).
int64_t solve_bytes(size_t N, size_t NI, size_t NE, size_t NC, int cap, int nvt, int ntiles, bool sums) {
    lssph_handle layout;
    layout.has_sums = sums;
    size_t total = 0;
    visit_solve_arrays(&layout, N, NI, NE, NC, cap, nvt, ntiles, [&](auto** p, size_t n) { total += array_bytes(p, n); });
    return (int64_t)total;
}

// Dynamic shared memory above 48 KB needs an opt-in per kernel; set once per
// instantiation while the handle is prepared (never during graph capture).
template <class K>
void smem_optin(K kernel) {
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tile_smem_bytes(64, 8, true));
}


// ---- kernel dispatch on lanes, register budget and precision ------------------------------
// The mixed-precision kernels exist for 2 and 4 lanes per particle.
// MX: 0 FP64, 1 mixed precision, 2 mixed precision with compensated pair sums.
template <int NB, int GG, int MX>
void run_stage(lssph_handle* h, const StageCfg& S, const Where& w) {
    if (h->classical) {   // SPH_MODEL 1 / 2 (FP64 only)
        if constexpr (!MX) {
            if (h->preparing) {
                smem_optin(k_stage_classical<NB, GG, false>);
                smem_optin(k_stage_classical<NB, GG, true>);
                return;
            }
            auto kern = h->tight ? k_stage_classical<NB, GG, true> : k_stage_classical<NB, GG, false>;
            launch_kernel_p(w.pdl, w.priority, kern, w.count, PPB * GG, h->smem_bytes, w.stream, h->P,
                            h->F[h->sb], h->F[h->sb ^ 1], h->L[h->lb], h->L[next_list(h->lb)], h->gstart, h->glist,
                            h->W, S, h->sc, h->ntx, w.tiles);
            h->launch_counter++;
        }
        return;
    }
    if (h->preparing) {
        smem_optin(k_stage<NB, GG, 0, MX>);
        smem_optin(k_stage<NB, GG, 1, MX>);
        smem_optin(k_stage<NB, GG, 2, MX>);
        return;
    }
    auto kern = h->tight ? k_stage<NB, GG, 1, MX> : k_stage<NB, GG, 0, MX>;
    if (h->budget == 2) kern = k_stage<NB, GG, 2, MX>;
    launch_kernel_p(w.pdl, w.priority, kern, w.count, PPB * GG, h->smem_bytes, w.stream, h->P, h->F[h->sb],
                    h->F[h->sb ^ 1], h->L[h->lb], h->L[next_list(h->lb)], h->gstart, h->glist, h->W, S, h->sc, h->ntx,
                    w.tiles);
    h->launch_counter++;
}

template <int NB>
void launch_stage(lssph_handle* h, const StageCfg& S, const Where& w) {
    ProfScope prof(h, LSSPH_KIND_STAGE);
    if (h->order >= 3) { launch_stage_hi(h, S, w.tiles, w.count, w.stream, w.pdl, w.priority); return; }
    if (h->mixed) {
        if (h->comp) {
            if (h->G == 2) run_stage<NB, 2, 2>(h, S, w);
            else run_stage<NB, 4, 2>(h, S, w);
        } else {
            if (h->G == 2) run_stage<NB, 2, 1>(h, S, w);
            else run_stage<NB, 4, 1>(h, S, w);
        }
        return;
    }
    switch (h->G) {
        case 1: run_stage<NB, 1, 0>(h, S, w); break;
        case 2: run_stage<NB, 2, 0>(h, S, w); break;
        case 8: run_stage<NB, 8, 0>(h, S, w); break;
        default: run_stage<NB, 4, 0>(h, S, w); break;
    }
}

// The stage kernel over the tiles of w.  In the split shape this is the pair kernel only:
// launch_stage_tail then runs the solve kernel once every tile of the stage is done.
void launch_stage_any(lssph_handle* h, const StageCfg& S, const Where& w) {
    if (h->split) { launch_stage_pairs(h, S, w); return; }
    if (h->nb_rhs == 1) launch_stage<1>(h, S, w);
    else if (h->nb_rhs == 5) launch_stage<5>(h, S, w);
    else launch_stage<4>(h, S, w);
}

void launch_stage_tail(lssph_handle* h, const StageCfg& S, bool pdl) {
    if (h->split) launch_stage_solve(h, S, h->stream, pdl);
}

// A whole stage (every tile, then the split shape's solve kernel).
void launch_stage_any(lssph_handle* h, const StageCfg& S) {
    launch_stage_any(h, S, all_tiles(h));
    launch_stage_tail(h, S, h->pdl);
}

// zero_list >= 0: clear that list's scatter counters (the list the preceding stage read).
template <int NB, int WQ>
void launch_ghost_t(lssph_handle* h, int zero_list, int reset_umax, cudaStream_t stream, bool pdl, int priority) {
    ProfScope prof(h, LSSPH_KIND_GHOST);
    const Fld& F = h->F[h->sb];
    const Lst& L = h->L[h->lb];
    const int G = h->Gg;
    const VMTiles VT{h->vt_tile, h->vt_start, h->vt_vm};
    int* zc = zero_list >= 0 ? h->L[zero_list].cnt : nullptr;
    const size_t sm = h->smem_ghost;
#define LSSPH_GHOST(GG)                                                                                    \
    if (h->preparing) { smem_optin(k_ghost<NB, GG, WQ>); return; }                                        \
    launch_kernel_p(pdl, priority, k_ghost<NB, GG, WQ>, h->nvt, PPB * GG, sm, stream, h->P, F, L, h->gstart, h->glist, h->V, VT, h->ntx, zc, \
                                                          reset_umax, h->sc)
    switch (G) {
        case 1: LSSPH_GHOST(1); break;
        case 2: LSSPH_GHOST(2); break;
        case 8: LSSPH_GHOST(8); break;
        default: LSSPH_GHOST(4); break;
    }
#undef LSSPH_GHOST
    h->launch_counter++;
}

template <int NB>
void launch_ghost_nb(lssph_handle* h, int zero_list, int reset_umax, cudaStream_t stream, bool pdl, int priority) {
    if (h->wq == 1) launch_ghost_t<NB, 1>(h, zero_list, reset_umax, stream, pdl, priority);
    else if (h->wq == 6) launch_ghost_t<NB, 6>(h, zero_list, reset_umax, stream, pdl, priority);
    else launch_ghost_t<NB, 3>(h, zero_list, reset_umax, stream, pdl, priority);
}

void launch_ghost_on(lssph_handle* h, int zero_list, int reset_umax, cudaStream_t stream, bool pdl,
                     int priority = 0) {
    if (h->num_ext == 0) {   // periodic domain: no ghosts, only the bookkeeping of the launch
        ProfScope prof(h, LSSPH_KIND_GHOST);
        if (h->preparing) return;
        const int nb = std::max(1, std::min(148, (h->grid.ncell + 255) / 256));
        int* zc = zero_list >= 0 ? h->L[zero_list].cnt : nullptr;
        launch_kernel_p(pdl, priority, k_housekeep, nb, 256, 0, stream, h->P, zc, reset_umax, h->sc);
        h->launch_counter++;
        return;
    }
    if (h->nb_ghost == 1) launch_ghost_nb<1>(h, zero_list, reset_umax, stream, pdl, priority);
    else if (h->nb_ghost == 4) launch_ghost_nb<4>(h, zero_list, reset_umax, stream, pdl, priority);
    else launch_ghost_nb<3>(h, zero_list, reset_umax, stream, pdl, priority);
}

void launch_ghost(lssph_handle* h, int zero_list = -1, int reset_umax = 0) {
    launch_ghost_on(h, zero_list, reset_umax, h->stream, h->pdl);
}

template <int NB, int GG, int MX>
void run_pst(lssph_handle* h, const Where& w) {
    if (h->classical) {   // first-order basis, q = 2 (shift_interpolate_mod.f90:43-44)
        if constexpr (!MX) {
            if (h->preparing) {
                smem_optin(k_pst<NB, GG, false, false, 1>);
                smem_optin(k_pst<NB, GG, true, false, 1>);
                return;
            }
            auto kern = h->tight ? k_pst<NB, GG, true, false, 1> : k_pst<NB, GG, false, false, 1>;
            launch_kernel_p(w.pdl, w.priority, kern, w.count, PPB * GG, h->smem_bytes, w.stream, h->P,
                            h->F[h->sb], h->F[h->sb ^ 1], h->L[h->lb], h->L[next_list(h->lb)], h->gstart, h->glist,
                            h->W, h->sc, h->ntx, w.tiles);
            h->launch_counter++;
        }
        return;
    }
    if (h->preparing) {
        smem_optin(k_pst<NB, GG, 0, MX>);
        smem_optin(k_pst<NB, GG, 1, MX>);
        smem_optin(k_pst<NB, GG, 2, MX>);
        return;
    }
    auto kern = h->tight ? k_pst<NB, GG, 1, MX> : k_pst<NB, GG, 0, MX>;
    if (h->budget == 2) kern = k_pst<NB, GG, 2, MX>;
    launch_kernel_p(w.pdl, w.priority, kern, w.count, PPB * GG, h->smem_bytes, w.stream, h->P, h->F[h->sb],
                    h->F[h->sb ^ 1], h->L[h->lb], h->L[next_list(h->lb)], h->gstart, h->glist, h->W, h->sc, h->ntx,
                    w.tiles);
    h->launch_counter++;
}

template <int NB>
void launch_pst_t(lssph_handle* h, const Where& w) {
    ProfScope prof(h, LSSPH_KIND_PST);
    if (h->order >= 3) { launch_pst_hi(h, w.tiles, w.count, w.stream, w.pdl, w.priority); return; }
    if (h->mixed) {
        if (h->comp) {
            if (h->G == 2) run_pst<NB, 2, 2>(h, w);
            else run_pst<NB, 4, 2>(h, w);
        } else {
            if (h->G == 2) run_pst<NB, 2, 1>(h, w);
            else run_pst<NB, 4, 1>(h, w);
        }
        return;
    }
    switch (h->G) {
        case 1: run_pst<NB, 1, 0>(h, w); break;
        case 2: run_pst<NB, 2, 0>(h, w); break;
        case 8: run_pst<NB, 8, 0>(h, w); break;
        default: run_pst<NB, 4, 0>(h, w); break;
    }
}

void launch_pst_any(lssph_handle* h, const Where& w) {
    if (h->split) { launch_pst_pairs(h, w); return; }
    if (h->has_tem) launch_pst_t<4>(h, w);
    else launch_pst_t<3>(h, w);
}

void launch_pst_tail(lssph_handle* h, bool pdl) {
    if (h->split) launch_pst_solve(h, h->stream, pdl);
}

// ---- operator sequences (enqueue only) -----------------------------------------------------
// One RK stage: RHS + update (+ scatter), cell list finish, ghost.
StageCfg stage_cfg(const lssph_handle* h, int stage, bool fused_step) {
    StageCfg S{};
    S.mode = MODE_STAGE;
    S.stage = stage;
    const double dt = h->p.dt;
    if (h->p.rk == 2) {
        S.last = stage == 2;
        S.dt2 = (stage == 1) ? dt / 2.0 : dt;
    } else {
        S.last = stage == 4;
        if (stage == 1) { S.dt1 = dt / 6.0; S.dt2 = dt / 2.0; }
        else if (stage == 2) { S.dt1 = dt / 3.0; S.dt2 = dt / 2.0; }
        else if (stage == 3) { S.dt1 = dt / 3.0; S.dt2 = dt; }
        else { S.dt1 = dt / 6.0; S.dt2 = 0.0; }
    }
    S.do_scatter = h->p1 ? 0 : 1;
    S.do_umax = (fused_step && h->pst_on) ? 1 : 0;
    S.do_steady = (fused_step && h->p1) ? 1 : 0;
    S.write_rhs = 1;
    return S;
}

void enq_stage(lssph_handle* h, int stage, bool fused_step) {
    launch_stage_any(h, stage_cfg(h, stage, fused_step));
    h->sb ^= 1;
    if (!h->p1) {
        h->lb = next_list(h->lb);
        launch_ghost(h, prev_list(h->lb), 0);   // also clears the list the stage just consumed
    } else {
        launch_ghost(h);
    }
}

void enq_pst(lssph_handle* h) {
    launch_pst_any(h, all_tiles(h));
    launch_pst_tail(h, h->pdl);
    h->sb ^= 1;
    h->lb = next_list(h->lb);
    launch_ghost(h, prev_list(h->lb), 1);
}

// Set the shared-memory opt-in of every kernel instantiation this handle launches.
void prepare_kernels(lssph_handle* h) {
    h->preparing = true;
    StageCfg S{};
    if (h->lanes_auto) {   // the other lane count the measurement may pick
        h->G = 2;
        launch_stage_any(h, S);
        launch_pst_any(h, all_tiles(h));
        h->G = 4;
    }
    launch_stage_any(h, S);
    launch_ghost(h);
    launch_pst_any(h, all_tiles(h));
    if (h->order >= 3 && !h->hi_fixed) {   // the other mapping the measurement may pick
        h->hi_thread = !h->hi_thread;
        launch_stage_any(h, S);
        launch_pst_any(h, all_tiles(h));
        h->hi_thread = !h->hi_thread;
    }
    if (split_capable(h)) {   // the split shape the measurement may pick
        launch_stage_pairs(h, S, all_tiles(h));
        launch_pst_pairs(h, all_tiles(h));
    }
    h->preparing = false;
}

void enq_epilogue(lssph_handle* h, bool pdl) {
    ProfScope prof(h, LSSPH_KIND_OTHER);
    launch_kernel(pdl, k_epilogue, 1, 1, 0, h->stream, h->P, h->sc);
    h->launch_counter++;
}

void enq_step(lssph_handle* h) {
    const int ns = h->p.rk == 2 ? 2 : 4;
    for (int s = 1; s <= ns; ++s) enq_stage(h, s, true);
    if (h->pst_on) enq_pst(h);
    if (h->p1) enq_epilogue(h, h->pdl);
}

// The same time step with each ghost launch beside the next stage's interior tiles
// (tiles whose halo holds no ghost particle need no ghost values).  On the side stream
// the ghost launch is followed by the wall tiles; both streams join before the next
// stage.  Every launch reads and writes exactly what it does in enq_step: the ghost
// launch touches ghost entries, virtual markers and the list two rotations back, the
// interior tiles read interior entries and the current list and write the next list and
// the other state buffer.  Stage 1 still follows the previous step's last ghost launch,
// which counts the step and applies the step budget.
void enq_step_overlap(lssph_handle* h) {
    const int ns = h->p.rk == 2 ? 2 : 4;
    // the ghost launch and the wall tiles are the critical path: their CTAs go first
    const Where interior{h->tile_int, h->n_int, h->stream, false, 0};
    const Where wall{h->tile_wall, h->n_wall, h->aux, h->pdl, h->high_priority};
    launch_stage_any(h, stage_cfg(h, 1, true));
    h->sb ^= 1;
    int zero = -1;
    if (!h->p1) {
        h->lb = next_list(h->lb);
        zero = prev_list(h->lb);
    }
    auto fork = [&]() {
        cudaEventRecord(h->fork_ev, h->stream);
        cudaStreamWaitEvent(h->aux, h->fork_ev, 0);
    };
    auto join = [&]() {
        cudaEventRecord(h->join_ev, h->aux);
        cudaStreamWaitEvent(h->stream, h->join_ev, 0);
    };
    for (int s = 2; s <= ns; ++s) {
        const StageCfg S = stage_cfg(h, s, true);
        fork();
        launch_ghost_on(h, zero, 0, h->aux, false, h->high_priority);
        launch_stage_any(h, S, interior);
        launch_stage_any(h, S, wall);
        join();
        launch_stage_tail(h, S, false);
        h->sb ^= 1;
        if (!h->p1) {
            h->lb = next_list(h->lb);
            zero = prev_list(h->lb);
        }
    }
    if (h->pst_on) {
        fork();
        launch_ghost_on(h, zero, 0, h->aux, false, h->high_priority);
        launch_pst_any(h, interior);
        launch_pst_any(h, wall);
        join();
        launch_pst_tail(h, false);
        h->sb ^= 1;
        h->lb = next_list(h->lb);
        launch_ghost_on(h, prev_list(h->lb), 1, h->stream, false);
    } else {
        launch_ghost_on(h, zero, 0, h->stream, false);
    }
    if (h->p1) enq_epilogue(h, h->pdl);
}

int sync_check(lssph_handle* h);

// The autotuner's picks, once per process for each solve configuration: every handle of
// the same configuration (problem, sizes, cell grid and tiles, model, kernel type, walls,
// precision, schedule, lanes asked for, shape or mapping restriction) takes the first one's lanes,
// shape and budget.  So two handles of one solve (a solve alone and as a batch member, a
// restart, serving requests of one size) sum in the same order, and a stream of requests
// of one size is measured once.
struct TuneKey {
    int64_t v[21];
    bool operator<(const TuneKey& o) const { return std::lexicographical_compare(v, v + 21, o.v, o.v + 21); }
};
struct TunePick {
    int G, budget;
    bool split, hi_thread;
    double us[3];
};
std::mutex g_tune_mu;
std::map<TuneKey, TunePick> g_tune_picks;

TuneKey tune_key(const lssph_handle* h, bool try_fused, bool try_split) {
    int dev = 0;
    cudaGetDevice(&dev);
    const lssph_params& p = h->p;
    return TuneKey{{dev, p.target_problem, h->num_int, h->num_ext, h->grid.nx, h->grid.ny, h->grid.cap, h->ntiles,
                    h->n_int, p.sph_model, p.kernel_type, p.wall_model, p.precision, p.rk, p.periodic, p.lanes,
                    h->overlap ? 1 : 0, h->pdl ? 1 : 0, try_fused ? 1 : 0, try_split ? 1 : 0,
                    h->hi_fixed ? (h->hi_thread ? 1 : 2) : 0}};
}

// Pick the lane count (lanes = 0), the kernel shape and the register budget of the stage
// and PST kernels by timing each option on the current state, keep the fastest.  Every
// option gives bit-identical results except the lane count, which changes sums at the
// rounding level.
int autotune(lssph_handle* h) {
    h->tuned = true;
    StageCfg S{};
    S.mode = MODE_RHS_ONLY;
    S.stage = 1;
    S.write_rhs = 1;
    const int64_t c0 = h->launch_counter;
    // level 2 (five CTAs per SM) exists for the q = 5 LS stage and PST kernels
    const int levels = (!h->classical && h->order == 2) ? 3 : 2;
    // the q = 5 LS kernels at 2 or 4 lanes may also run split (pair kernel, then solve
    // kernel): budget levels 0-4 of the pair kernel.  LSSPH_KERNEL_SHAPE = fused / split
    // restricts the choice.
    const char* shape = std::getenv("LSSPH_KERNEL_SHAPE");
    const bool can_split = split_capable(h);
    const bool try_fused = !(can_split && shape && std::strcmp(shape, "split") == 0);
    const bool try_split = can_split && !(shape && std::strcmp(shape, "fused") == 0);
    // LSSPH_REGISTER_BUDGET = loose / tight / five (/ six / eight: the split shape's 768 and
    // 1024 threads per SM): skip the timing
    const char* force = std::getenv("LSSPH_REGISTER_BUDGET");
    if (force) {
        static const char* const names[5] = {"loose", "tight", "five", "six", "eight"};
        int level = -1;
        for (int t = 0; t < 5; ++t)
            if (std::strcmp(force, names[t]) == 0) level = t;
        if (level >= 0) {
            h->split = !try_fused;
            h->budget = std::min(level, h->split ? 4 : levels - 1);
            h->tight = h->budget >= 1;
            return LSSPH_OK;
        }
    }
    const TuneKey key = tune_key(h, try_fused, try_split);
    // held for the whole measurement, so that a second handle of the same configuration
    // (on another thread) waits and takes this pick instead of measuring its own
    std::unique_lock<std::mutex> tune_lock(g_tune_mu);
    {
        const auto it = g_tune_picks.find(key);
        if (it != g_tune_picks.end()) {
            const TunePick& k = it->second;
            h->G = k.G;
            h->split = k.split;
            h->hi_thread = k.hi_thread;
            h->budget = k.budget;
            h->tight = k.budget >= 1;
            for (int t = 0; t < 3; ++t) h->tune_us[t] = k.us[t];
            return LSSPH_OK;
        }
    }
    // lanes = 0 on a q = 5 LS solve: 4 lanes per particle unless 2 lanes run the RHS
    // pass at least 5 % faster (the margin keeps the pick, and with it the summation order,
    // the same from run to run when the two are close).  The shape and the budget change no
    // result, so they go to the fastest.
    //
    // One timed pass is a whole time step (enq_step, or enq_step_overlap in the overlapped
    // schedule) run on the solve's own state and undone afterwards: the solve's device block
    // is copied aside first and copied back after every option, with the host-side buffer
    // parities, so the measurement leaves no trace.  The RHS pass alone misjudged the
    // overlapped closed box by about 10 % in both directions (the ghost launches beside the
    // interior tiles, the split shape's solve kernel after the join, the update and scatter
    // the RHS pass leaves out).  Without device memory for the copy, the pass is the RHS
    // over every tile (then the split shape's solve kernel), which writes only the RHS.
    const int sb0 = h->sb, lb0 = h->lb;
    const size_t block_bytes = (size_t)h->alloc_bytes;
    void* saved = nullptr;
    const bool by_steps = cudaMalloc(&saved, block_bytes) == cudaSuccess;
    if (!by_steps) cudaGetLastError();   // no room: clear the error, time RHS passes
    struct FreeOnExit {   // an error return below still releases the copy
        void*& p;
        ~FreeOnExit() {
            if (p) cudaFree(p);
        }
    } free_on_exit{saved};
    if (by_steps)
        CUDA_TRY(h, cudaMemcpyAsync(saved, h->block, block_bytes, cudaMemcpyDeviceToDevice, h->stream));
    auto pass = [&]() {
        if (!by_steps) launch_stage_any(h, S);
        else if (h->overlap) enq_step_overlap(h);
        else enq_step(h);
    };
    // A solve that a step budget or the steady state has stopped would time no-op steps:
    // the measured steps run with both lifted (the copy puts them back).
    auto lift_stops = [&]() -> cudaError_t {
        if (!by_steps) return cudaSuccess;
        cudaError_t e = cudaMemsetAsync(&h->sc->steady, 0, sizeof(int), h->stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(&h->sc->step_limit, 0, 2 * sizeof(int), h->stream);
        return e;
    };
    auto restore = [&]() -> cudaError_t {
        h->sb = sb0;
        h->lb = lb0;
        return by_steps ? cudaMemcpyAsync(h->block, saved, block_bytes, cudaMemcpyDeviceToDevice, h->stream)
                        : cudaSuccess;
    };
    const int nlanes = h->lanes_auto ? 2 : 1;
    const int lane_opts[2] = {h->G, 2};
    // option t: fused at budget t (t < levels), split at budget t - levels.  The higher-
    // order kernels (SPH_MODEL 4-6) have one register budget and two mappings instead:
    // t = 0 thread per particle over a cell tile, t = 1 warp per particle.
    const bool hi = h->order >= 3;
    const bool hi_free = hi && !h->hi_fixed;
    constexpr int kOpts = 3 + 5;
    const int nopt = hi ? (hi_free ? 2 : 1) : levels + (try_split ? 5 : 0);
    double us[2][kOpts];
    for (auto& row : us)
        for (double& v : row) v = 1e30;
    // Every option is timed in each of several interleaved rounds and keeps its fastest
    // round, so that a clock ramp or a neighbour's burst during one round does not decide
    // the pick (a single round swung the choice by about 10 % between machines).
    const int kRounds = by_steps ? 3 : 5;
    for (int round = 0; round < kRounds; ++round) {
        for (int g = 0; g < nlanes; ++g) {
            h->G = lane_opts[g];
            for (int t = 0; t < nopt; ++t) {
                if (hi) {
                    if (hi_free) h->hi_thread = t == 0;
                    h->split = false;
                    h->budget = 0;
                } else {
                    h->split = t >= levels;
                    if (!h->split && !try_fused) continue;
                    h->budget = h->split ? t - levels : t;
                }
                h->tight = h->budget >= 1;
                CUDA_TRY(h, lift_stops());
                pass();   // warm-up (instruction cache, L2)
                CUDA_TRY(h, cudaEventRecord(h->ev0, h->stream));
                for (int r = 0; r < 3; ++r) pass();
                CUDA_TRY(h, cudaEventRecord(h->ev1, h->stream));
                CUDA_TRY(h, cudaEventSynchronize(h->ev1));
                float ms = 0.f;
                CUDA_TRY(h, cudaEventElapsedTime(&ms, h->ev0, h->ev1));
                us[g][t] = std::min(us[g][t], 1e3 * ms / 3.0);
                CUDA_TRY(h, restore());
            }
        }
    }
    int best_t[2] = {0, 0};
    for (int g = 0; g < nlanes; ++g) {
        // In the overlapped step the interior tiles share the SMs with the ghost launch: the
        // fused kernels at four CTAs per SM (the tight budget) leave room for it where three
        // do not, so the overlapped step's fused kernels take the tight budget (the split
        // shape's pair kernels fit more CTAs per SM at any level).
        best_t[g] = hi ? 0 : (try_fused ? (h->overlap ? 1 : 0) : levels + 1);
        for (int t = 0; t < nopt; ++t) {
            if (!hi && h->overlap && t < levels && t != 1) continue;
            if (us[g][t] < us[g][best_t[g]]) best_t[g] = t;
        }
        // The fused loose budget only when it beats the tight one by more than 3 %: the
        // measurement runs warm steps, and where the two are that close in them, cold-cache
        // steps ran tight faster (periodic Taylor-Green 128^2: 102 against 111 us per step
        // with the L2 flushed before each step, within 1-2 % of each other warm).
        if (!hi && best_t[g] == 0 && try_fused && us[g][1] <= 1.03 * us[g][0]) best_t[g] = 1;
    }
    if (by_steps) {
        CUDA_TRY(h, cudaStreamSynchronize(h->stream));
        const cudaError_t e = cudaFree(saved);
        saved = nullptr;
        CUDA_TRY(h, e);
    }
    const int pick = (nlanes == 2 && us[1][best_t[1]] < 0.95 * us[0][best_t[0]]) ? 1 : 0;
    h->G = lane_opts[pick];
    for (int t = 0; t < 3; ++t) h->tune_us[t] = (t < levels && us[pick][t] < 1e29) ? us[pick][t] : 0.0;
    if (hi) {
        if (hi_free) h->hi_thread = best_t[pick] == 0;
        h->split = false;
        h->budget = 0;
    } else {
        h->split = best_t[pick] >= levels;
        h->budget = h->split ? best_t[pick] - levels : best_t[pick];
    }
    h->tight = h->budget >= 1;
    h->launch_counter = c0;
    const int rc = sync_check(h);
    if (rc == LSSPH_OK)
        g_tune_picks.emplace(key, TunePick{h->G, h->budget, h->split, h->hi_thread,
                                           {h->tune_us[0], h->tune_us[1], h->tune_us[2]}});
    return rc;
}

// The handle's own launches use the measured register budget; batches choose per group
// and never need it, so the measurement waits for the first solo launch.
int ensure_tuned(lssph_handle* h) { return h->tuned ? LSSPH_OK : autotune(h); }

}  // namespace

int lssph::resolve_lanes(lssph_handle* h) { return (h->lanes_auto && !h->tuned) ? autotune(h) : LSSPH_OK; }

bool lssph::pdl_enabled() {
    const char* v = std::getenv("LSSPH_PDL");
    return !(v && std::strcmp(v, "0") == 0);
}

namespace {

int check_scalars(lssph_handle* h, Scalars* out) {
    Scalars s{};
    if (h->sc_host) {   // one copy into pinned memory behind the queued work, one sync
        CUDA_TRY(h, cudaMemcpyAsync(h->sc_host, h->sc, sizeof(Scalars), cudaMemcpyDeviceToHost, h->stream));
        CUDA_TRY(h, cudaStreamSynchronize(h->stream));
        s = *h->sc_host;
    } else {
        CUDA_TRY(h, cudaStreamSynchronize(h->stream));
        CUDA_TRY(h, cudaMemcpy(&s, h->sc, sizeof(Scalars), cudaMemcpyDeviceToHost));
    }
    if (out) *out = s;
    // a NaN position also leaves the grid: report the root cause first
    if (s.err & ERR_NONFINITE) return fail(h, LSSPH_E_NONFINITE, "a non-finite value appeared in the particle state");
    if (s.err & ERR_OUT_OF_DOMAIN) return fail(h, LSSPH_E_OUT_OF_DOMAIN, "a particle left the cell grid");
    if (s.err & ERR_CELL_OVERFLOW) return fail(h, LSSPH_E_CELL_OVERFLOW, "a cell holds more particles than its slot capacity");
    return LSSPH_OK;
}

int sync_check(lssph_handle* h) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(h, LSSPH_E_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
    return check_scalars(h, nullptr);
}

// The launches of nsteps time steps behind whatever is queued on the handle's stream (graph
// replays, captured on first use per parity), no synchronisation.  finish_steps reads the
// scalars back (one synchronisation) and puts the buffer parities where the last executed
// step left them.
struct StepMark {
    int64_t launches0;
    int sb_start, lb_start;
};

int enqueue_steps(lssph_handle* h, int32_t nsteps, StepMark* mark) {
    mark->launches0 = h->launch_counter;
    mark->sb_start = h->sb;
    mark->lb_start = h->lb;
    // The step count at entry, recorded on the device behind the queued work, in place of a
    // read-back before the launches: every kernel of a halted solve (steady state -- where
    // the reference leaves its time loop --, step budget, error) does nothing, so the one
    // read-back after the launches tells how many steps ran and why they stopped.
    CUDA_TRY(h, cudaMemcpyAsync(&h->sc->step_mark, &h->sc->step_count, sizeof(int), cudaMemcpyDeviceToDevice,
                                h->stream));
    CUDA_TRY(h, cudaEventRecord(h->ev0, h->stream));
    for (int st = 0; st < nsteps; ++st) {
        cudaGraphExec_t& ge = h->graph[h->sb][h->lb];
        if (!ge) {
            const int sb0 = h->sb, lb0 = h->lb;
            const int64_t c0 = h->launch_counter;
            CUDA_TRY(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
            if (h->overlap) enq_step_overlap(h);
            else enq_step(h);
            cudaGraph_t g = nullptr;
            CUDA_TRY(h, cudaStreamEndCapture(h->stream, &g));
            // per-node priorities: the overlapped step's critical path runs first
            const cudaError_t e = cudaGraphInstantiate(&ge, g, cudaGraphInstantiateFlagUseNodePriority);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) return fail(h, LSSPH_E_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
            h->graph_launches = (int)(h->launch_counter - c0);
            h->launch_counter = c0;
            h->step_sbf = h->sb ^ sb0;
            h->step_lba = (h->lb - lb0 + kLists) % kLists;
            h->sb = sb0;
            h->lb = lb0;
        }
        CUDA_TRY(h, cudaGraphLaunch(ge, h->stream));
        h->launch_counter += h->graph_launches;
        h->sb ^= h->step_sbf;
        h->lb = (h->lb + h->step_lba) % kLists;
    }
    CUDA_TRY(h, cudaEventRecord(h->ev1, h->stream));
    return LSSPH_OK;
}

// executed: the steps that ran (nsteps unless the solve stopped on the way).
int finish_steps(lssph_handle* h, int32_t nsteps, const StepMark& mark, int32_t* steady_step_out, int* executed) {
    Scalars s1{};
    const int rc = check_scalars(h, &s1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    h->last_ms = ms;
    h->last_launches = h->launch_counter - mark.launches0;
    // steps after a stop (steady state, step budget, error) ran as no-ops: the buffers
    // sit where the last executed step left them
    *executed = s1.step_count - s1.step_mark;
    if (*executed != nsteps) {
        h->sb = mark.sb_start ^ (h->step_sbf & *executed & 1);
        h->lb = (mark.lb_start + h->step_lba * *executed) % kLists;
    }
    if (rc != LSSPH_OK) return rc;
    if (s1.steady && steady_step_out && s1.steady_step > s1.step_mark) *steady_step_out = s1.steady_step - s1.step_mark;
    return LSSPH_OK;
}

// Mixed precision: the split-precision positions of the current state, both buffers.
void write_split_pos(lssph_handle* h) {
    if (!h->P.split_pos) return;
    k_split_pos<<<blocks_for(std::max(h->num_int, h->grid.ncell), 128), 128, 0, h->stream>>>(
        h->P, h->F[h->sb], h->F[h->sb ^ 1], h->W.key, h->gstart, h->glist);
}

// Build the cell list of the current positions into list buffer lb (fresh).
int rebuild_cells(lssph_handle* h) {
    static_assert(kLists == 3, "k_clear_counts zeroes three lists");
    k_clear_counts<<<blocks_for(h->grid.ncell, 256), 256, 0, h->stream>>>(h->L[0].cnt, h->L[1].cnt, h->L[2].cnt,
                                                                          h->grid.ncell);
    k_scatter<<<blocks_for(h->num_int, 128), 128, 0, h->stream>>>(h->P, h->F[h->sb], h->L[h->lb], h->gstart, h->W.key, h->sc);
    write_split_pos(h);
    return LSSPH_OK;
}

// Device address of a caller's host buffer of `bytes` that the GPU can read and write
// directly (page-locked and mapped, e.g. from cudaHostAlloc or cudaHostRegister: both its
// first and its last byte), else nullptr (ordinary pageable memory goes through copies).
void* mapped_host(const void* p, size_t bytes) {
    if (!p || bytes == 0) return nullptr;
    cudaPointerAttributes a{}, b{};
    const char* last = static_cast<const char*>(p) + (bytes - 1);
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess || cudaPointerGetAttributes(&b, last) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    if (a.type != cudaMemoryTypeHost || b.type != cudaMemoryTypeHost || !a.devicePointer || !b.devicePointer)
        return nullptr;
    if (static_cast<char*>(b.devicePointer) != static_cast<char*>(a.devicePointer) + (bytes - 1)) return nullptr;
    return a.devicePointer;
}

// Access flags of the current device on host memory p (cuPointerGetAttribute with
// CU_POINTER_ATTRIBUTE_ACCESS_FLAGS, reached through the runtime's driver entry point so
// that the library does not link libcuda), or -1 when the driver cannot be asked.
long long host_access_flags(const void* p) {
    static_assert(CU_POINTER_ATTRIBUTE_ACCESS_FLAG_READ == kAccessRead &&
                  CU_POINTER_ATTRIBUTE_ACCESS_FLAG_READWRITE == kAccessReadWrite, "access flag values");
    static const PFN_cuPointerGetAttribute_v4000 fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuPointerGetAttribute", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return reinterpret_cast<PFN_cuPointerGetAttribute_v4000>(f);
    }();
    if (!fn) return -1;
    unsigned long long flags = 0;   // the driver writes a 32-bit enum into the low bytes
    if (fn(&flags, CU_POINTER_ATTRIBUTE_ACCESS_FLAGS, (CUdeviceptr)(uintptr_t)p) != CUDA_SUCCESS) return -1;
    return (long long)(flags & 0xffffffffull);
}

// Every non-null field mapped (and, for a kernel that stores into them, writable from the
// device at both ends): device addresses into out[0..6], true.
bool all_mapped(const double* const (&f)[7], size_t bytes, double* (&out)[7], bool store = false) {
    for (int k = 0; k < 7; ++k) {
        out[k] = nullptr;
        if (!f[k]) continue;
        out[k] = static_cast<double*>(mapped_host(f[k], bytes));
        if (!out[k]) return false;
        if (store && !(mapped_store_allowed(host_access_flags(f[k])) &&
                       mapped_store_allowed(host_access_flags(reinterpret_cast<const char*>(f[k]) + bytes - 1))))
            return false;
    }
    return true;
}

// The copies (or, into page-locked mapped buffers the device may write, one kernel) of the
// current state into caller-owned host arrays, queued on the handle's stream: the caller
// synchronises before reading them.  tem of a solve without temperature is zeroed here.
int enqueue_download(lssph_handle* h, int32_t* ptype, double* x, double* y, double* u, double* v, double* rho,
                     double* pre, double* tem) {
    const size_t bytes = sizeof(double) * (size_t)h->num_total;
    const Fld& F = h->F[h->sb];
    if (tem && !h->has_tem) std::memset(tem, 0, bytes);
    if (ptype) std::memcpy(ptype, h->ptype.data(), sizeof(int32_t) * h->num_total);
    {   // page-locked, mapped host buffers: one kernel writes them
        const double* const f[7] = {x, y, u, v, rho, pre, h->has_tem ? tem : nullptr};
        double* d[7];
        if (all_mapped(f, bytes, d, true)) {
            k_download_mapped<<<blocks_for(h->num_total, 256), 256, 0, h->stream>>>(
                h->P, F, HostOut{d[0], d[1], d[2], d[3], d[4], d[5], d[6]});
            CUDA_TRY(h, cudaGetLastError());
            return LSSPH_OK;
        }
    }
    if (x) CUDA_TRY(h, cudaMemcpyAsync(x, F.x, bytes, cudaMemcpyDeviceToHost, h->stream));
    if (y) CUDA_TRY(h, cudaMemcpyAsync(y, F.y, bytes, cudaMemcpyDeviceToHost, h->stream));
    if (u) CUDA_TRY(h, cudaMemcpyAsync(u, F.u, bytes, cudaMemcpyDeviceToHost, h->stream));
    if (v) CUDA_TRY(h, cudaMemcpyAsync(v, F.v, bytes, cudaMemcpyDeviceToHost, h->stream));
    if (rho) CUDA_TRY(h, cudaMemcpyAsync(rho, F.rho, bytes, cudaMemcpyDeviceToHost, h->stream));
    if (pre) CUDA_TRY(h, cudaMemcpyAsync(pre, F.pre, bytes, cudaMemcpyDeviceToHost, h->stream));
    if (tem && h->has_tem) CUDA_TRY(h, cudaMemcpyAsync(tem, F.tem, bytes, cudaMemcpyDeviceToHost, h->stream));
    return LSSPH_OK;
}

// The current buffer gets every particle.  On a later upload (both = false) the other buffer
// needs the ghost particles only: the next stage (or PST) writes every interior field of it
// before anything reads it -- except in problem 1, whose stages write u alone, so there it
// gets every particle too.  Page-locked, mapped host buffers are read by one kernel.
int upload_fields(lssph_handle* h, const double* x, const double* y, const double* u, const double* v,
                  const double* rho, const double* pre, const double* tem, bool both = true) {
    {
        const double* const f[7] = {x, y, u, v, rho, pre, h->has_tem ? tem : nullptr};
        double* d[7];
        if (all_mapped(f, sizeof(double) * (size_t)h->num_total, d)) {
            const int first_b = (both || h->p1) ? 0 : h->num_int;
            k_upload_mapped<<<blocks_for(h->num_total, 256), 256, 0, h->stream>>>(
                h->P, h->F[h->sb], h->F[h->sb ^ 1], HostFld{d[0], d[1], d[2], d[3], d[4], d[5], d[6]}, first_b);
            return LSSPH_OK;
        }
    }
    for (int b = 0; b < 2; ++b) {
        const Fld& F = h->F[b];
        const size_t first = (both || b == h->sb || h->p1) ? 0 : (size_t)h->num_int;
        const size_t n = (size_t)h->num_total - first;
        if (n == 0) continue;
        const size_t bytes = sizeof(double) * n;
        if (x) CUDA_TRY(h, cudaMemcpyAsync(F.x + first, x + first, bytes, cudaMemcpyHostToDevice, h->stream));
        if (y) CUDA_TRY(h, cudaMemcpyAsync(F.y + first, y + first, bytes, cudaMemcpyHostToDevice, h->stream));
        if (u) CUDA_TRY(h, cudaMemcpyAsync(F.u + first, u + first, bytes, cudaMemcpyHostToDevice, h->stream));
        if (v) CUDA_TRY(h, cudaMemcpyAsync(F.v + first, v + first, bytes, cudaMemcpyHostToDevice, h->stream));
        if (rho) CUDA_TRY(h, cudaMemcpyAsync(F.rho + first, rho + first, bytes, cudaMemcpyHostToDevice, h->stream));
        if (pre) CUDA_TRY(h, cudaMemcpyAsync(F.pre + first, pre + first, bytes, cudaMemcpyHostToDevice, h->stream));
        if (tem && h->has_tem)
            CUDA_TRY(h, cudaMemcpyAsync(F.tem + first, tem + first, bytes, cudaMemcpyHostToDevice, h->stream));
        k_volume<<<blocks_for(h->num_total, 128), 128, 0, h->stream>>>(h->P, F);
    }
    return LSSPH_OK;
}

// Solve blocks come from the device's default stream-ordered memory pool, which keeps freed
// blocks for reuse (release threshold at its maximum): a destroy then frees with
// cudaFreeAsync on the solve's own stream instead of cudaFree, which synchronised the whole
// device and now and then took a good fraction of a second in a serving loop that creates
// and destroys solves while batch calls run.  lssph_mem_info trims the pool first, so the
// free memory it reports still counts freed blocks as free.
cudaError_t pool_for_blocks(cudaMemPool_t* pool) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if ((e = cudaDeviceGetDefaultMemPool(pool, dev)) != cudaSuccess) return e;
    static std::mutex mu;
    static bool configured[64] = {};
    std::lock_guard<std::mutex> lock(mu);
    if (dev >= 0 && dev < 64 && !configured[dev]) {
        uint64_t keep = UINT64_MAX;
        if ((e = cudaMemPoolSetAttribute(*pool, cudaMemPoolAttrReleaseThreshold, &keep)) != cudaSuccess) return e;
        configured[dev] = true;
    }
    return cudaSuccess;
}

void free_handle(lssph_handle* h) {
    if (!h) return;
    if (h->batch) batch_forget(h->batch, h);
    if (h->stream) cudaStreamSynchronize(h->stream);
    snapshot_release(h);
    postproc_release(h);
    for (auto& row : h->graph)
        for (auto& g : row)
            if (g) cudaGraphExecDestroy(g);
    if (h->block) {
        cudaFreeAsync(h->block, h->stream);
        cudaStreamSynchronize(h->stream);
    }
    return_pinned_slot(h->sc_host);
    for (cudaEvent_t e : h->prof_events) cudaEventDestroy(e);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->fork_ev) cudaEventDestroy(h->fork_ev);
    if (h->join_ev) cudaEventDestroy(h->join_ev);
    if (h->aux) cudaStreamDestroy(h->aux);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

int create_impl(const lssph_params* pin, int num_total, int num_int, const int32_t* ptype, const double* x,
                const double* y, const double* u, const double* v, const double* rho, const double* pre,
                const double* tem, lssph_handle** out) {
    std::string msg;
    if (!pin || !ptype || !x || !y || !u || !v || !rho || !pre || !out) return fail(nullptr, LSSPH_E_BAD_PARAM, "null argument");
    *out = nullptr;
    if (check_param(pin, &msg) != LSSPH_OK) return fail(nullptr, LSSPH_E_BAD_PARAM, msg);
    if (pin->sph_model < 1 || pin->sph_model > 6)
        return fail(nullptr, LSSPH_E_UNSUPPORTED, "SPH_MODEL must be between 1 and 6");
    const bool mixed = pin->precision == LSSPH_PRECISION_MIXED || pin->precision == LSSPH_PRECISION_MIXED_COMPENSATED;
    if (pin->sph_model != 3 && mixed)
        return fail(nullptr, LSSPH_E_UNSUPPORTED, "mixed precision runs the LS-SPH model (SPH_MODEL 3) only");
    if (pin->precision != LSSPH_PRECISION_FP64 && !mixed)
        return fail(nullptr, LSSPH_E_BAD_PARAM,
                    "precision must be LSSPH_PRECISION_FP64, LSSPH_PRECISION_MIXED or LSSPH_PRECISION_MIXED_COMPENSATED");
    if (mixed && pin->lanes != 0 && pin->lanes != 2 && pin->lanes != 4)
        return fail(nullptr, LSSPH_E_UNSUPPORTED, "mixed precision runs with 2 or 4 lanes per particle (lanes = 0, 2 or 4)");
    if (pin->target_problem == 4 && !tem) return fail(nullptr, LSSPH_E_BAD_PARAM, "tem required for problem 4");
    if (num_int <= 0 || num_total < num_int || (num_total == num_int && !pin->periodic))
        return fail(nullptr, LSSPH_E_BAD_PARAM, "bad particle counts");
    if (pin->periodic && num_total != num_int)
        return fail(nullptr, LSSPH_E_BAD_PARAM, "a periodic domain has no ghost particles (num_total == num_int)");
    for (int i = 0; i < num_total; ++i) {
        if ((i < num_int) != (ptype[i] == 0))
            return fail(nullptr, LSSPH_E_BAD_PARAM, "ptype must be 0 for the first num_int particles and 1..8 after");
    }
    lssph_handle* h = new lssph_handle();
    h->p = *pin;
    init_param(&h->p);
    h->num_total = num_total;
    h->num_int = num_int;
    h->num_ext = num_total - num_int;
    h->problem = h->p.target_problem;
    h->has_tem = h->problem == 4;
    h->p1 = h->problem == 1;
    h->pst_on = h->problem != 1;   // main.f90:132-134
    h->nb_rhs = h->p1 ? 1 : (h->has_tem ? 5 : 4);
    h->nb_ghost = h->p1 ? 1 : (h->has_tem ? 4 : 3);
    h->wq = h->p.wall_model == 1 ? 1 : (h->p.wall_model == 3 ? 6 : 3);
    h->mixed = h->p.precision != LSSPH_PRECISION_FP64;
    h->comp = h->p.precision == LSSPH_PRECISION_MIXED_COMPENSATED;
    h->classical = h->p.sph_model <= 2;
    h->order = h->p.sph_model >= 4 ? h->p.sph_model - 1 : 2;   // LSSPH_A_mod.f90:46-56
    h->has_sums = split_sums(h->p);
    {
        // Higher-order kernel shape, measured on B200 (Taylor-Green 128^2 / 256^2, closed
        // box and periodic): thread per particle is faster for q = 9 (1.5-1.6x) and q = 14
        // (1.04-1.6x), warp per particle for q = 20 (1.7-1.8x), where the thread's shared-
        // memory slot leaves too few warps per SM.  LSSPH_HI_KERNEL=thread|warp overrides.
        // That is the starting choice; the autotuner times both mappings on the solve itself
        // at its first launch and keeps the faster (both give identical results).
        const char* v = std::getenv("LSSPH_HI_KERNEL");
        h->hi_thread = h->order <= 4;
        h->hi_fixed = v && (std::strcmp(v, "warp") == 0 || std::strcmp(v, "thread") == 0);
        if (v && std::strcmp(v, "warp") == 0) h->hi_thread = false;
        if (v && std::strcmp(v, "thread") == 0) h->hi_thread = true;
    }
    h->pdl = pdl_enabled();
    {
        int least = 0, greatest = 0;
        if (cudaDeviceGetStreamPriorityRange(&least, &greatest) == cudaSuccess) h->high_priority = greatest;
    }
    {
        const char* v = std::getenv("LSSPH_OVERLAP");   // 0: ghost launches run alone
        h->overlap_allowed = !(v && std::strcmp(v, "0") == 0);
    }
    h->G = h->p.lanes > 0 ? h->p.lanes : 4;
    h->Gg = h->p.lanes > 0 ? h->p.lanes : 4;
    h->ptype.assign(ptype, ptype + num_total);

    int rc = build_virtual_markers(&h->p, num_total, num_int, ptype, x, y, &h->vm, &msg);
    if (rc == LSSPH_OK) rc = build_cell_grid(&h->p, num_total, num_int, x, y, h->vm, &h->grid, &msg);
    if (rc != LSSPH_OK) { free_handle(h); return fail(nullptr, rc, msg); }

    // ---- constants ----
    const lssph_params& p = h->p;
    Phys& P = h->P;
    P.problem = p.target_problem; P.kt = p.kernel_type; P.rk = p.rk; P.wall_model = p.wall_model;
    P.sph_model = p.sph_model;
    P.periodic = p.periodic;
    P.Lx = p.len_x;
    P.u_bc_top = p.u_bc_top; P.u_bc_bottom = p.u_bc_bottom; P.u_bc_left = p.u_bc_left; P.u_bc_right = p.u_bc_right;
    P.tem_bc_top = p.tem_bc_top; P.tem_bc_bottom = p.tem_bc_bottom; P.tem_bc_left = p.tem_bc_left;
    P.tem_bc_right = p.tem_bc_right;
    P.nx = h->grid.nx; P.ny = h->grid.ny; P.ncell = h->grid.ncell; P.cap = h->grid.cap;
    P.num_total = num_total; P.num_int = num_int; P.num_ext = h->num_ext;
    P.u_top = p.u_top; P.tem_top = p.tem_top; P.tem_bottom = p.tem_bottom; P.tem_left = p.tem_left;
    P.tem_right = p.tem_right;
    P.h = p.h;
    P.ih1 = 1.0 / p.h;
    P.ih2A = P.ih1 / p.h;          // inv_h(2) = inv_h(1)/h  (LSSPH_A_mod.f90:90-93)
    P.ih2B = P.ih1 * P.ih1;        // inv_h2 = inv_h*inv_h  (interpolate_LSSPH_B_mod.f90:151-152)
    P.h_eff_sq = p.h_eff * p.h_eff;
    P.inv_h_eff = p.periodic ? h->grid.inv_cw : 1.0 / p.h_eff;   // cell keys
    P.cw = p.periodic ? p.len_x / (double)h->grid.nx : p.h_eff;    // cell origins
    P.split_pos = h->mixed ? 1 : 0;
    P.SP_mass = p.SP_mass;
    P.W_ave = p.W_ave;
    P.wnorm = kernel_norm(p.kernel_type, p.h);
    P.dt = p.dt;
    P.c_sq = p.sound_speed * p.sound_speed;
    P.rho_ref = p.rho_ref;
    P.vis_ref = p.vis_ref;
    P.delta = ((p.coe_delta_sph * p.sound_speed) * p.h) * p.zeta_RSST;
    P.zeta_sq = p.zeta_RSST * p.zeta_RSST;
    P.xi_sq = p.xi_VIM * p.xi_VIM;
    P.alpha_ref = p.alpha_ref;
    P.gravity = p.gravity;
    P.tem_ave = p.tem_ave;
    P.thermal_dif = p.thermal_dif;
    P.PST_c = p.PST_c;
    P.threshold = p.threshold;
    P.hydro_coef_top = ((p.rho_ref * p.alpha_ref) * (p.tem_top - p.tem_ave)) * p.gravity;
    P.hydro_coef_bottom = ((p.rho_ref * p.alpha_ref) * (p.tem_bottom - p.tem_ave)) * p.gravity;
    P.iWave = 1.0 / p.W_ave;
    P.izeta2 = 1.0 / (p.zeta_RSST * p.zeta_RSST);
    P.ixi2 = 1.0 / (p.xi_VIM * p.xi_VIM);
    P.m3h = -3.0 / p.h;
    P.m5h = -5.0 / p.h;

    // ---- device memory ----
    auto cu = [&](cudaError_t e) { return e == cudaSuccess ? LSSPH_OK : fail(nullptr, LSSPH_E_CUDA, cudaGetErrorString(e)); };
    if ((rc = cu(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking))) != LSSPH_OK ||
        (rc = cu(cudaStreamCreateWithFlags(&h->aux, cudaStreamNonBlocking))) != LSSPH_OK ||
        (rc = cu(cudaEventCreateWithFlags(&h->fork_ev, cudaEventDisableTiming))) != LSSPH_OK ||
        (rc = cu(cudaEventCreateWithFlags(&h->join_ev, cudaEventDisableTiming))) != LSSPH_OK ||
        (rc = cu(cudaEventCreate(&h->ev0))) != LSSPH_OK || (rc = cu(cudaEventCreate(&h->ev1))) != LSSPH_OK) {
        free_handle(h);
        return rc;
    }
    const size_t N = num_total, NI = num_int, NE = h->num_ext, NC = h->grid.ncell;
    // cell tiles and the tiles that hold virtual markers (grouped, ascending marker id)
    h->ntx = (h->grid.nx + TX - 1) / TX;
    h->nty = (h->grid.ny + TY - 1) / TY;
    h->ntiles = h->ntx * h->nty;
    h->smem_bytes = h->mixed ? tile_smem_bytes_mx(h->grid.cap, h->G, h->has_tem)
                             : tile_smem_bytes(h->grid.cap, h->G, h->has_tem);
    h->smem_ghost = tile_smem_bytes(h->grid.cap, h->Gg, h->has_tem);   // ghosts stay FP64
    std::vector<int32_t> vt_tile, vt_start, vt_vm;
    vm_chunks(h->grid, h->ntx, h->ntiles, &vt_tile, &vt_start, &vt_vm);
    h->nvt = (int)vt_tile.size();
    // tiles whose halo holds no ghost particle (interior) and the others (wall)
    std::vector<int32_t> t_int, t_wall;
    for (int t = 0; t < h->ntiles; ++t) {
        const int cx0 = (t % h->ntx) * TX - 1, cy0 = (t / h->ntx) * TY - 1;
        bool interior = true;
        for (int hy = 0; hy < HY && interior; ++hy)
            for (int hx = 0; hx < HX && interior; ++hx) {
                const int cx = cx0 + hx, cy = cy0 + hy;
                if (cx < 0 || cx >= h->grid.nx || cy < 0 || cy >= h->grid.ny) { interior = false; break; }
                const int c = cx + cy * h->grid.nx;
                if (h->grid.gstart[c + 1] != h->grid.gstart[c]) interior = false;
            }
        (interior ? t_int : t_wall).push_back(t);
    }
    h->n_int = (int)t_int.size();
    h->n_wall = (int)t_wall.size();
    h->overlap = h->overlap_allowed && h->n_int > 0 && h->n_wall > 0 && !p.periodic;
    // lanes = 0: the first solo launch measures 2 and 4 lanes (q = 5 LS in FP64 or mixed
    // precision) and keeps the faster; the shared memory covers both
    h->lanes_auto = h->p.lanes == 0 && !h->classical && h->order == 2;
    if (h->lanes_auto)
        h->smem_bytes = std::max(h->smem_bytes, h->mixed ? tile_smem_bytes_mx(h->grid.cap, 2, h->has_tem)
                                                         : tile_smem_bytes(h->grid.cap, 2, h->has_tem));
    // one device block for every array of the solve (one allocation from the stream-ordered
    // pool on the solve's stream, freed the same way)
    const size_t block = (size_t)solve_bytes(N, NI, NE, NC, h->grid.cap, h->nvt, h->ntiles, h->has_sums);
    {
        // pinned scalar copy target (optional: without it the checks copy through pageable memory)
        h->sc_host = pinned_slot();
        cudaMemPool_t pool;
        cudaError_t e = pool_for_blocks(&pool);
        if (e == cudaSuccess) e = cudaMallocFromPoolAsync(&h->block, block, pool, h->stream);
        // a pooled block may hold an earlier solve's data: every array starts at zero (the
        // arrays a problem never writes, e.g. the v and rho RHS of problem 1, read as zeros)
        if (e == cudaSuccess) e = cudaMemsetAsync(h->block, 0, block, h->stream);
        if (e != cudaSuccess) {
            h->block = nullptr;
            free_handle(h);
            return fail(nullptr, LSSPH_E_CUDA, std::string("cudaMallocFromPoolAsync: ") + cudaGetErrorString(e));
        }
        h->alloc_bytes = (int64_t)block;
        size_t off = 0;
        char* base = static_cast<char*>(h->block);
        visit_solve_arrays(h, N, NI, NE, NC, h->grid.cap, h->nvt, h->ntiles, [&](auto** p, size_t n) {
            using T = std::remove_reference_t<decltype(**p)>;
            *p = reinterpret_cast<T*>(base + off);
            off += array_bytes(p, n);
        });
    }
    bool ok = true;
    Work& W = h->W;
    VMd& V = h->V;

    // ---- host-side constant arrays ----
    std::vector<double> src(NI, 0.0), K(NE, 0.0), zeros(std::max(NI, NE), 0.0), ones(NI, 1.0);
    std::vector<int32_t> mode(NE, XM_NEG);
    if (h->p1 && !p.periodic) {   // the periodic problem 1 is source-free (src stays 0.0)
        for (size_t i = 0; i < NI; ++i)   // LSSPH_A_mod.f90:247-248 (positions never move in problem 1)
            src[i] = ((2.0 * (kPi * kPi)) * std::sin(kPi * (x[i] - p.WL_thick))) * std::cos(kPi * (y[i] - p.WL_thick));
        for (size_t me = 0; me < NE; ++me) {   // extrapolate_diff_test_mod.f90:40-103
            const int t = h->vm.ptype[me];
            const double vx = h->vm.x[me], vy = h->vm.y[me], xg = x[num_int + me];
            if (t == 1) {
                if (p.u_bc_bottom == 1) mode[me] = XM_COPY;
                else { mode[me] = XM_K_MINUS; K[me] = 2.0 * std::sin(kPi * (vx - p.WL_thick)); }
            } else if (t == 2) {
                if (p.u_bc_top == 1) mode[me] = XM_COPY;
                else { mode[me] = XM_K_MINUS; K[me] = 2.0 * (-std::sin(kPi * (vx - p.WL_thick))); }
            } else if (t == 3) {
                if (p.u_bc_left == 1) { mode[me] = XM_PLUS_K; K[me] = (kPi * std::cos(kPi * (vy - p.WL_thick))) * (xg - vx); }
                else mode[me] = XM_NEG;
            } else if (t == 4) {
                if (p.u_bc_right == 1) { mode[me] = XM_PLUS_K; K[me] = ((-kPi) * std::cos(kPi * (vy - p.WL_thick))) * (xg - vx); }
                else mode[me] = XM_NEG;
            } else {
                mode[me] = XM_NEG;
            }
        }
    }
    auto H2D = [&](void* dst, const void* srcp, size_t bytes) {
        if (ok && bytes && cudaMemcpyAsync(dst, srcp, bytes, cudaMemcpyHostToDevice, h->stream) != cudaSuccess) ok = false;
    };
    H2D(W.src, src.data(), sizeof(double) * NI);
    H2D(W.f_prev, ones.data(), sizeof(double) * NI);   // setup_closed_box_mod.f90:160-163
    H2D(V.x, h->vm.x.data(), sizeof(double) * NE);
    H2D(V.y, h->vm.y.data(), sizeof(double) * NE);
    H2D(V.nx, h->vm.nx.data(), sizeof(double) * NE);
    H2D(V.ny, h->vm.ny.data(), sizeof(double) * NE);
    H2D(V.ptype, h->vm.ptype.data(), sizeof(int32_t) * NE);
    H2D(V.key, h->grid.vm_key.data(), sizeof(int32_t) * NE);
    H2D(V.K, K.data(), sizeof(double) * NE);
    H2D(V.mode, mode.data(), sizeof(int32_t) * NE);
    H2D(V.u, zeros.data(), sizeof(double) * NE);
    H2D(V.v, zeros.data(), sizeof(double) * NE);
    H2D(V.pre, zeros.data(), sizeof(double) * NE);
    H2D(V.tem, zeros.data(), sizeof(double) * NE);
    H2D(h->gstart, h->grid.gstart.data(), sizeof(int32_t) * (NC + 1));
    H2D(h->glist, h->grid.glist.data(), sizeof(int32_t) * NE);
    H2D(h->vt_tile, vt_tile.data(), sizeof(int32_t) * vt_tile.size());
    H2D(h->vt_start, vt_start.data(), sizeof(int32_t) * vt_start.size());
    H2D(h->vt_vm, vt_vm.data(), sizeof(int32_t) * NE);
    H2D(h->tile_int, t_int.data(), sizeof(int32_t) * t_int.size());
    H2D(h->tile_wall, t_wall.data(), sizeof(int32_t) * t_wall.size());
    if (ok && cudaMemsetAsync(h->sc, 0, sizeof(Scalars), h->stream) != cudaSuccess) ok = false;
    if (ok && cudaMemsetAsync(W.key, 0, sizeof(int32_t) * NI, h->stream) != cudaSuccess) ok = false;
    for (int b = 0; b < 2 && ok; ++b)
        if (cudaMemsetAsync(h->F[b].tem, 0, sizeof(double) * N, h->stream) != cudaSuccess) ok = false;
    for (int b = 0; b < kLists && ok; ++b)
        if (cudaMemsetAsync(h->L[b].slots, 0xff, sizeof(int) * NC * h->grid.cap, h->stream) != cudaSuccess) ok = false;
    if (!ok) { free_handle(h); return fail(nullptr, LSSPH_E_CUDA, "device initialisation failed"); }
    prepare_kernels(h);
    if ((rc = upload_fields(h, x, y, u, v, rho, pre, tem)) != LSSPH_OK ||
        (rc = rebuild_cells(h)) != LSSPH_OK || (rc = sync_check(h)) != LSSPH_OK) {
        const std::string m = h->err;
        free_handle(h);
        return fail(nullptr, rc, m);
    }
    *out = h;
    return LSSPH_OK;
}

}  // namespace

// =====================================================================================
// C ABI (handle half)
// =====================================================================================
extern "C" {

int lssph_create(const lssph_params* p, int32_t num_total, int32_t num_int, const int32_t* ptype,
                 const double* x, const double* y, const double* u, const double* v, const double* rho,
                 const double* pre, const double* tem, lssph_handle** out) {
    return create_impl(p, num_total, num_int, ptype, x, y, u, v, rho, pre, tem, out);
}

void lssph_destroy(lssph_handle* h) { free_handle(h); }

const char* lssph_handle_error(const lssph_handle* h) { return h ? h->err.c_str() : "null handle"; }

int lssph_get_params(const lssph_handle* h, lssph_params* out) {
    if (!h || !out) return fail(nullptr, LSSPH_E_BAD_PARAM, "null argument");
    *out = h->p;
    return LSSPH_OK;
}

int lssph_counts(const lssph_handle* h, int32_t* num_total, int32_t* num_int, int32_t* num_ext, int32_t* num_cells) {
    if (!h) return fail(nullptr, LSSPH_E_BAD_PARAM, "null handle");
    if (num_total) *num_total = h->num_total;
    if (num_int) *num_int = h->num_int;
    if (num_ext) *num_ext = h->num_ext;
    if (num_cells) *num_cells = h->grid.ncell;
    return LSSPH_OK;
}

int lssph_calculate_rhs(lssph_handle* h) {
    if (!h) return fail(nullptr, LSSPH_E_BAD_PARAM, "null handle");
    if (const int rc_t = ensure_tuned(h)) return rc_t;
    StageCfg S{};
    S.mode = MODE_RHS_ONLY;
    S.stage = 1;
    S.write_rhs = 1;
    launch_stage_any(h, S);
    return sync_check(h);
}

int lssph_update_cell(lssph_handle* h) {
    if (!h) return fail(nullptr, LSSPH_E_BAD_PARAM, "null handle");
    CUDA_TRY(h, cudaMemsetAsync(h->L[next_list(h->lb)].cnt, 0, sizeof(int) * h->grid.ncell, h->stream));
    k_scatter<<<blocks_for(h->num_int, 128), 128, 0, h->stream>>>(h->P, h->F[h->sb], h->L[next_list(h->lb)], h->gstart,
                                                                     h->W.key, h->sc);
    write_split_pos(h);
    h->lb = next_list(h->lb);
    CUDA_TRY(h, cudaMemsetAsync(h->L[prev_list(h->lb)].cnt, 0, sizeof(int) * h->grid.ncell, h->stream));
    return sync_check(h);
}

int lssph_ghost(lssph_handle* h) {
    if (!h) return fail(nullptr, LSSPH_E_BAD_PARAM, "null handle");
    launch_ghost(h);
    return sync_check(h);
}

int lssph_rk2(lssph_handle* h) {
    if (!h) return fail(nullptr, LSSPH_E_BAD_PARAM, "null handle");
    if (const int rc_t = ensure_tuned(h)) return rc_t;
    if (h->p.rk != 2) return fail(h, LSSPH_E_BAD_PARAM, "handle was configured with RK = 4");
    for (int s = 1; s <= 2; ++s) enq_stage(h, s, false);
    return sync_check(h);
}

int lssph_rk4(lssph_handle* h) {
    if (!h) return fail(nullptr, LSSPH_E_BAD_PARAM, "null handle");
    if (const int rc_t = ensure_tuned(h)) return rc_t;
    if (h->p.rk != 4) return fail(h, LSSPH_E_BAD_PARAM, "handle was configured with RK = 2");
    for (int s = 1; s <= 4; ++s) enq_stage(h, s, false);
    return sync_check(h);
}

int lssph_pst(lssph_handle* h) {
    if (!h) return fail(nullptr, LSSPH_E_BAD_PARAM, "null handle");
    if (const int rc_t = ensure_tuned(h)) return rc_t;
    CUDA_TRY(h, cudaMemsetAsync(&h->sc->umax2, 0, sizeof(unsigned long long), h->stream));
    k_umax<<<blocks_for(h->num_int, 128), 128, 0, h->stream>>>(h->P, h->F[h->sb], h->sc);
    enq_pst(h);
    return sync_check(h);
}

int lssph_check_steady_state(lssph_handle* h, int32_t* is_steady) {
    if (!h || !is_steady) return fail(nullptr, LSSPH_E_BAD_PARAM, "null argument");
    CUDA_TRY(h, cudaMemsetAsync(&h->sc->dfmax, 0, sizeof(unsigned long long), h->stream));
    k_steady_max<<<blocks_for(h->num_int, 128), 128, 0, h->stream>>>(h->P, h->F[h->sb], h->W, h->sc);
    Scalars s{};
    int rc = check_scalars(h, &s);
    if (rc != LSSPH_OK) return rc;
    double df;
    std::memcpy(&df, &s.dfmax, sizeof(df));
    *is_steady = (df < h->p.threshold) ? 1 : 0;
    if (!*is_steady) k_copy_fprev<<<blocks_for(h->num_int, 128), 128, 0, h->stream>>>(h->P, h->F[h->sb], h->W);
    CUDA_TRY(h, cudaMemsetAsync(&h->sc->dfmax, 0, sizeof(unsigned long long), h->stream));
    return sync_check(h);
}

int lssph_step(lssph_handle* h, int32_t nsteps, int32_t* steady_step_out) {
    if (!h) return fail(nullptr, LSSPH_E_BAD_PARAM, "null handle");
    if (steady_step_out) *steady_step_out = 0;
    if (nsteps <= 0) return LSSPH_OK;
    int rc = ensure_tuned(h);
    if (rc != LSSPH_OK) return rc;
    StepMark mark{};
    if ((rc = enqueue_steps(h, nsteps, &mark)) != LSSPH_OK) return rc;
    int executed = 0;
    return finish_steps(h, nsteps, mark, steady_step_out, &executed);
}

int lssph_mem_info(int64_t* free_bytes, int64_t* total_bytes) {
    size_t f = 0, t = 0;
    cudaMemPool_t pool;
    if (pool_for_blocks(&pool) == cudaSuccess) cudaMemPoolTrimTo(pool, 0);   // freed blocks count as free
    cudaGetLastError();
    const cudaError_t err = cudaMemGetInfo(&f, &t);
    if (err != cudaSuccess) return fail(nullptr, LSSPH_E_CUDA, std::string("cudaMemGetInfo: ") + cudaGetErrorString(err));
    if (free_bytes) *free_bytes = (int64_t)f;
    if (total_bytes) *total_bytes = (int64_t)t;
    return LSSPH_OK;
}

int lssph_device_bytes(const lssph_handle* h, int64_t* bytes) {
    if (!h || !bytes) return fail(nullptr, LSSPH_E_BAD_PARAM, "null argument");
    *bytes = h->alloc_bytes;
    return LSSPH_OK;
}

int lssph_estimate_device_bytes(const lssph_params* pin, int64_t* bytes) {
    if (!pin || !bytes) return fail(nullptr, LSSPH_E_BAD_PARAM, "null argument");
    std::string msg;
    lssph_params p = *pin;
    init_param(&p);
    if (check_param(&p, &msg) != LSSPH_OK) return fail(nullptr, LSSPH_E_BAD_PARAM, msg);
    int nt = 0, ni = 0;
    int rc = closed_box_counts(&p, &nt, &ni);
    if (rc != LSSPH_OK) return fail(nullptr, rc, "bad particle counts");
    std::vector<int32_t> ptype(nt);
    std::vector<double> x(nt), y(nt), u(nt), v(nt), rho(nt), pre(nt), tem(nt);
    rc = setup_particles(&p, nt, ptype.data(), x.data(), y.data(), u.data(), v.data(), rho.data(), pre.data(),
                         tem.data(), &msg);
    VirtualMarkers vm;
    CellGrid grid;
    if (rc == LSSPH_OK) rc = build_virtual_markers(&p, nt, ni, ptype.data(), x.data(), y.data(), &vm, &msg);
    if (rc == LSSPH_OK) rc = build_cell_grid(&p, nt, ni, x.data(), y.data(), vm, &grid, &msg);
    if (rc != LSSPH_OK) return fail(nullptr, rc, msg);
    const int ntx = (grid.nx + TX - 1) / TX, nty = (grid.ny + TY - 1) / TY;
    std::vector<int32_t> vt_tile, vt_start, vt_vm;
    vm_chunks(grid, ntx, ntx * nty, &vt_tile, &vt_start, &vt_vm);
    *bytes = solve_bytes(nt, ni, nt - ni, grid.ncell, grid.cap, (int)vt_tile.size(), ntx * nty, split_sums(p));
    return LSSPH_OK;
}

int lssph_get_schedule(const lssph_handle* h, int32_t* tiles, int32_t* interior_tiles, int32_t* overlapped) {
    if (!h) return fail(nullptr, LSSPH_E_BAD_PARAM, "null handle");
    if (tiles) *tiles = h->ntiles;
    if (interior_tiles) *interior_tiles = h->n_int;
    if (overlapped) *overlapped = h->overlap ? 1 : 0;
    return LSSPH_OK;
}

int lssph_set_step_budget(lssph_handle* h, int32_t nsteps) {
    if (!h) return fail(nullptr, LSSPH_E_BAD_PARAM, "null handle");
    if (nsteps < 0) return fail(h, LSSPH_E_BAD_PARAM, "the step budget must be >= 0");
    Scalars s{};
    int rc = check_scalars(h, &s);
    if (rc != LSSPH_OK) return rc;
    s.step_limit = nsteps > 0 ? s.step_count + nsteps : 0;
    s.done = 0;
    CUDA_TRY(h, cudaMemcpy(&h->sc->step_limit, &s.step_limit, 2 * sizeof(int), cudaMemcpyHostToDevice));
    return LSSPH_OK;
}

int lssph_get_progress(lssph_handle* h, int32_t* steps_done, int32_t* stopped) {
    if (!h) return fail(nullptr, LSSPH_E_BAD_PARAM, "null handle");
    Scalars s{};
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    CUDA_TRY(h, cudaMemcpy(&s, h->sc, sizeof(Scalars), cudaMemcpyDeviceToHost));
    if (steps_done) *steps_done = s.step_count;
    if (stopped) *stopped = s.steady ? 1 : (s.done ? 2 : 0);
    return LSSPH_OK;
}

int lssph_upload(lssph_handle* h, const double* x, const double* y, const double* u, const double* v,
                 const double* rho, const double* pre, const double* tem) {
    if (!h) return fail(nullptr, LSSPH_E_BAD_PARAM, "null handle");
    int rc = upload_fields(h, x, y, u, v, rho, pre, tem, false);
    if (rc != LSSPH_OK) return rc;
    if (!h->p1 && (x || y)) {
        if ((rc = rebuild_cells(h)) != LSSPH_OK) return rc;
    }
    return sync_check(h);
}

int lssph_download(lssph_handle* h, int32_t* ptype, double* x, double* y, double* u, double* v, double* rho,
                   double* pre, double* tem) {
    if (!h) return fail(nullptr, LSSPH_E_BAD_PARAM, "null handle");
    const int rc = enqueue_download(h, ptype, x, y, u, v, rho, pre, tem);
    if (rc != LSSPH_OK) return rc;
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    return LSSPH_OK;
}

int lssph_advance_host(lssph_handle* h, int32_t nsteps, double* x, double* y, double* u, double* v, double* rho,
                       double* pre, double* tem, int32_t* steady_step_out) {
    if (!h) return fail(nullptr, LSSPH_E_BAD_PARAM, "null handle");
    if (!x || !y || !u || !v || !rho || !pre || (h->has_tem && !tem))
        return fail(h, LSSPH_E_BAD_PARAM, "lssph_advance_host: null state array");
    if (steady_step_out) *steady_step_out = 0;
    if (nsteps < 0) return fail(h, LSSPH_E_BAD_PARAM, "lssph_advance_host: nsteps must be >= 0");
    int rc = ensure_tuned(h);   // first call only: measures lanes / register budget
    if (rc != LSSPH_OK) return rc;
    // upload (as lssph_upload), steps (as lssph_step), download (as lssph_download), queued
    // back to back on the handle's stream; the scalar read-back is the one synchronisation
    if ((rc = upload_fields(h, x, y, u, v, rho, pre, tem, false)) != LSSPH_OK) return rc;
    if (!h->p1 && (rc = rebuild_cells(h)) != LSSPH_OK) return rc;
    StepMark mark{};
    if (nsteps > 0 && (rc = enqueue_steps(h, nsteps, &mark)) != LSSPH_OK) return rc;
    const int sb_queued = h->sb;
    if ((rc = enqueue_download(h, nullptr, x, y, u, v, rho, pre, h->has_tem ? tem : nullptr)) != LSSPH_OK) return rc;
    CUDA_TRY(h, cudaGetLastError());
    if (nsteps == 0) return sync_check(h);
    int executed = 0;
    rc = finish_steps(h, nsteps, mark, steady_step_out, &executed);
    // a solve that stopped on the way (steady state, step budget, error) sits in the other
    // buffer when it ran an odd number of steps fewer: read that one instead
    if (h->sb != sb_queued) {
        const int rc2 = enqueue_download(h, nullptr, x, y, u, v, rho, pre, h->has_tem ? tem : nullptr);
        if (rc2 != LSSPH_OK) return rc2;
        CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    }
    return rc;
}

int lssph_download_rhs(lssph_handle* h, double* ru, double* rv, double* rr, double* rt) {
    if (!h) return fail(nullptr, LSSPH_E_BAD_PARAM, "null handle");
    const size_t bytes = sizeof(double) * (size_t)h->num_int;
    if (ru) CUDA_TRY(h, cudaMemcpyAsync(ru, h->W.rhs_u, bytes, cudaMemcpyDeviceToHost, h->stream));
    if (rv) CUDA_TRY(h, cudaMemcpyAsync(rv, h->W.rhs_v, bytes, cudaMemcpyDeviceToHost, h->stream));
    if (rr) CUDA_TRY(h, cudaMemcpyAsync(rr, h->W.rhs_rho, bytes, cudaMemcpyDeviceToHost, h->stream));
    if (rt) CUDA_TRY(h, cudaMemcpyAsync(rt, h->W.rhs_tem, bytes, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    return LSSPH_OK;
}

int lssph_download_vm(lssph_handle* h, int32_t* ptype, double* x, double* y, double* u, double* v, double* pre,
                      double* tem) {
    if (!h) return fail(nullptr, LSSPH_E_BAD_PARAM, "null handle");
    const size_t ne = h->num_ext, bytes = sizeof(double) * ne;
    if (ptype) std::memcpy(ptype, h->vm.ptype.data(), sizeof(int32_t) * ne);
    if (x) std::memcpy(x, h->vm.x.data(), bytes);
    if (y) std::memcpy(y, h->vm.y.data(), bytes);
    if (u) CUDA_TRY(h, cudaMemcpyAsync(u, h->V.u, bytes, cudaMemcpyDeviceToHost, h->stream));
    if (v) CUDA_TRY(h, cudaMemcpyAsync(v, h->V.v, bytes, cudaMemcpyDeviceToHost, h->stream));
    if (pre) CUDA_TRY(h, cudaMemcpyAsync(pre, h->V.pre, bytes, cudaMemcpyDeviceToHost, h->stream));
    if (tem) CUDA_TRY(h, cudaMemcpyAsync(tem, h->V.tem, bytes, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    return LSSPH_OK;
}

int lssph_neighbors_csr(lssph_handle* h, int32_t which, int32_t* offsets, int32_t* idx, int64_t cap, int64_t* nnz_out) {
    if (!h || !offsets) return fail(nullptr, LSSPH_E_BAD_PARAM, "null argument");
    const int n = which == 0 ? h->num_int : h->num_ext;
    const int stride = 9 * h->grid.cap;
    int *d_out = nullptr, *d_cnt = nullptr;
    CUDA_TRY(h, cudaMallocAsync((void**)&d_out, sizeof(int) * (size_t)n * stride, h->stream));
    CUDA_TRY(h, cudaMallocAsync((void**)&d_cnt, sizeof(int) * (size_t)n, h->stream));
    k_neighbors<<<blocks_for(n, 128), 128, 0, h->stream>>>(h->P, h->F[h->sb], h->L[h->lb], h->gstart, h->glist,
                                                           h->W.key, h->V, which, stride, d_out, d_cnt);
    std::vector<int> out((size_t)n * stride), cnt(n);
    CUDA_TRY(h, cudaMemcpyAsync(out.data(), d_out, sizeof(int) * out.size(), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaMemcpyAsync(cnt.data(), d_cnt, sizeof(int) * cnt.size(), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaFreeAsync(d_out, h->stream));
    CUDA_TRY(h, cudaFreeAsync(d_cnt, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    int64_t nnz = 0;
    for (int i = 0; i < n; ++i) {
        offsets[i] = (int32_t)nnz;
        const int c = std::min(cnt[i], stride);
        std::sort(out.begin() + (size_t)i * stride, out.begin() + (size_t)i * stride + c);
        if (idx) {
            if (nnz + c > cap) return fail(h, LSSPH_E_CAPACITY, "neighbour index buffer too small");
            std::memcpy(idx + nnz, out.data() + (size_t)i * stride, sizeof(int32_t) * c);
        }
        nnz += c;
    }
    offsets[n] = (int32_t)nnz;
    if (nnz_out) *nnz_out = nnz;
    return LSSPH_OK;
}

int lssph_write_data(lssph_handle* h, const char* results_root, int32_t step) {
    if (!h || !results_root) return fail(nullptr, LSSPH_E_BAD_PARAM, "null argument");
    const size_t n = h->num_total;
    std::vector<int32_t> pt(n);
    std::vector<double> x(n), y(n), u(n), v(n), rho(n), pre(n), tem(n);
    int rc = lssph_download(h, pt.data(), x.data(), y.data(), u.data(), v.data(), rho.data(), pre.data(), tem.data());
    if (rc != LSSPH_OK) return rc;
    const std::string dir = std::string(results_root) + "/" + h->p.save_name + "/data";
    if (make_dirs(dir) != LSSPH_OK) return fail(h, LSSPH_E_IO, "cannot create " + dir);
    std::string msg;
    rc = write_data_file(dir + "/" + std::to_string(step) + ".dat", (int)n, h->has_tem, pt.data(), x.data(), y.data(),
                         u.data(), v.data(), rho.data(), pre.data(), tem.data(), &msg);
    return rc == LSSPH_OK ? rc : fail(h, rc, msg);
}

int lssph_write_param(lssph_handle* h, const char* results_root, const char* config_h_path) {
    if (!h || !results_root) return fail(nullptr, LSSPH_E_BAD_PARAM, "null argument");
    const std::string base = std::string(results_root) + "/" + h->p.save_name;
    const std::string cfg = base + "/config", dat = base + "/data";
    if (make_dirs(cfg) != LSSPH_OK || make_dirs(dat) != LSSPH_OK) return fail(h, LSSPH_E_IO, "cannot create " + base);
    if (config_h_path && config_h_path[0] && copy_file(config_h_path, cfg + "/config.h") != LSSPH_OK)
        return fail(h, LSSPH_E_IO, std::string("cannot copy ") + config_h_path);
    std::string msg;
    int rc = write_parameters_csv(cfg + "/parameters.csv", &h->p, h->num_total, h->num_int, h->num_ext, &msg);
    if (rc != LSSPH_OK) return fail(h, rc, msg);
    // cell_idx.dat: 1-based cell ids after init_cell + update_cell (write_param_mod.f90:133-136)
    std::vector<int32_t> key(h->num_int), cell(h->num_total);
    CUDA_TRY(h, cudaMemcpy(key.data(), h->W.key, sizeof(int32_t) * h->num_int, cudaMemcpyDeviceToHost));
    for (int i = 0; i < h->num_int; ++i) cell[i] = key[i] + 1;
    for (int me = 0; me < h->num_ext; ++me) cell[h->num_int + me] = h->grid.ghost_key[me] + 1;
    FILE* f = std::fopen((dat + "/cell_idx.dat").c_str(), "wb");
    if (!f) return fail(h, LSSPH_E_IO, "cannot open cell_idx.dat");
    const bool ok1 = std::fwrite(cell.data(), sizeof(int32_t), cell.size(), f) == cell.size();
    std::fclose(f);
    if (!ok1) return fail(h, LSSPH_E_IO, "short write to cell_idx.dat");
    // ghost() then VM.dat (write_param_mod.f90:141-159)
    if ((rc = lssph_ghost(h)) != LSSPH_OK) return rc;
    const size_t ne = h->num_ext;
    std::vector<int32_t> pt(ne);
    std::vector<double> vx(ne), vy(ne), vu(ne), vv(ne), vp(ne), vt(ne);
    if ((rc = lssph_download_vm(h, pt.data(), vx.data(), vy.data(), vu.data(), vv.data(), vp.data(), vt.data())) != LSSPH_OK)
        return rc;
    f = std::fopen((dat + "/VM.dat").c_str(), "wb");
    if (!f) return fail(h, LSSPH_E_IO, "cannot open VM.dat");
    bool ok = std::fwrite(pt.data(), sizeof(int32_t), ne, f) == ne;
    for (const auto* a : {&vx, &vy, &vu, &vv, &vp}) ok = ok && std::fwrite(a->data(), sizeof(double), ne, f) == ne;
    if (h->has_tem) ok = ok && std::fwrite(vt.data(), sizeof(double), ne, f) == ne;
    std::fclose(f);
    if (!ok) return fail(h, LSSPH_E_IO, "short write to VM.dat");
    return LSSPH_OK;
}

int lssph_step_profiled(lssph_handle* h, int32_t nsteps, double* ms_by_kind, int64_t* launches_by_kind) {
    if (!h || !ms_by_kind || !launches_by_kind) return fail(nullptr, LSSPH_E_BAD_PARAM, "null argument");
    if (const int rc_t = ensure_tuned(h)) return rc_t;
    for (int k = 0; k < LSSPH_KIND_COUNT; ++k) { ms_by_kind[k] = 0.0; launches_by_kind[k] = 0; }
    int rc = check_scalars(h, nullptr);
    if (rc != LSSPH_OK) return rc;
    h->profiling = true;
    h->prof_next = 0;
    h->prof_kinds.clear();
    for (int st = 0; st < nsteps; ++st) enq_step(h);
    h->profiling = false;
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    for (size_t k = 0; k < h->prof_kinds.size(); ++k) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, h->prof_events[2 * k], h->prof_events[2 * k + 1]);
        ms_by_kind[h->prof_kinds[k]] += ms;
        launches_by_kind[h->prof_kinds[k]] += 1;
    }
    return check_scalars(h, nullptr);
}

int lssph_get_tuning(const lssph_handle* hc, int32_t* lanes, int32_t* tight, double* rhs_us_loose,
                     double* rhs_us_tight) {
    if (!hc) return fail(nullptr, LSSPH_E_BAD_PARAM, "null handle");
    lssph_handle* h = const_cast<lssph_handle*>(hc);   // the measurement is a cache
    if (const int rc = ensure_tuned(h)) return rc;
    if (lanes) *lanes = h->G;
    if (tight) *tight = h->budget;
    if (rhs_us_loose) *rhs_us_loose = h->tune_us[0];
    if (rhs_us_tight) *rhs_us_tight = h->tune_us[1];
    return LSSPH_OK;
}

int lssph_get_kernel_shape(const lssph_handle* hc, int32_t* split) {
    if (!hc || !split) return fail(nullptr, LSSPH_E_BAD_PARAM, "null argument");
    lssph_handle* h = const_cast<lssph_handle*>(hc);   // the measurement is a cache
    if (const int rc = ensure_tuned(h)) return rc;
    *split = h->order >= 3 ? (h->hi_thread ? 2 : 3) : (h->split ? 1 : 0);
    return LSSPH_OK;
}

int lssph_last_step_stats(const lssph_handle* h, double* device_ms, int64_t* kernel_launches) {
    if (!h) return fail(nullptr, LSSPH_E_BAD_PARAM, "null handle");
    if (device_ms) *device_ms = h->last_ms;
    if (kernel_launches) *kernel_launches = h->last_launches;
    return LSSPH_OK;
}

}  // extern "C"
