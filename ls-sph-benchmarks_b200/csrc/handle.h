// handle.h -- the device state of one solve (lssph_handle), shared by the single-solve
// entry points (engine.cu) and the batched time loop (batch.cu).  Internal header.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <utility>
#include <vector>

#include "engine.h"
#include "kernels.cuh"

namespace lssph {
struct SnapState;   // asynchronous snapshots (snapshot.cu)
struct PPScratch;   // post-processing stream and scratch (postproc.cu)
}

struct lssph_handle {

    lssph_params p{};
    int num_total = 0, num_int = 0, num_ext = 0;
    int problem = 0;
    bool has_tem = false, p1 = false, pst_on = false;
    int nb_rhs = 4, nb_ghost = 3, nb_pst = 3, wq = 3;
    int G = 4, Gg = 4;
    bool mixed = false;                 // FP32 pair phase, FP64 solve + refinement
    bool comp = false;                  // mixed precision with compensated (Kahan) FP32 pair sums
    bool split = false;                 // q = 5 LS stage/PST: pair and solve kernels apart (autotuned)
    bool has_sums = false;              // Work::sums allocated (the split shape may run)
    bool classical = false;             // SPH_MODEL 1 / 2: kernel-gradient sums, q = 2 PST basis
    int order = 2;                      // Taylor order k of the LS basis (SPH_MODEL 3: 2; 4 / 5 / 6: 3 / 4 / 5)
    bool hi_thread = false;             // order >= 3: thread per particle (else warp per particle)
    bool hi_fixed = false;              // the mapping is fixed by LSSPH_HI_KERNEL (else autotuned)
    bool pdl = true;                    // programmatic dependent launches in the time step
    bool tuned = false;                 // register budget measured (first solo launch)
    bool lanes_auto = false;            // lanes = 0 on an FP64 q = 5 LS solve: 2 or 4 by measurement
    bool tight = false;                 // register budget of stage/PST kernels (autotuned): 4 CTAs/SM or more
    int budget = 0;                     // 0 loose, 1 tight (4 CTAs/SM), 2 five CTAs/SM; the split
                                        // shape's pair kernel also 3 (768 threads/SM), 4 (1024)
    double tune_us[3] = {0.0, 0.0, 0.0};   // RHS pass time per budget level
    lssph::CellGrid grid;
    lssph::VirtualMarkers vm;
    std::vector<int32_t> ptype;
    lssph::Phys P{};
    cudaStream_t stream = nullptr;
    cudaStream_t aux = nullptr;         // side stream of the overlapped time step
    cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
    int* tile_int = nullptr;            // tiles whose halo holds no ghost particle
    int* tile_wall = nullptr;           // the other tiles
    int n_int = 0, n_wall = 0;
    bool overlap_allowed = true;        // LSSPH_OVERLAP=0 turns the overlapped step off
    bool overlap = false;               // ghost launches run beside interior tiles
    int high_priority = 0;              // the device's highest launch priority (ghost + wall tiles)
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    void* block = nullptr;              // the one device allocation all arrays live in
    int64_t alloc_bytes = 0;            // its size
    lssph::Fld F[2]{};
    lssph::Lst L[lssph::kLists]{};      // cell lists in rotation: read one, scatter into the next
    lssph::Work W{};
    lssph::VMd V{};
    int* gstart = nullptr;
    int* glist = nullptr;
    int ntx = 0, nty = 0, ntiles = 0;   // cell tiles
    int nvt = 0;                        // tiles holding virtual markers
    int *vt_tile = nullptr, *vt_start = nullptr, *vt_vm = nullptr;
    size_t smem_bytes = 0;              // dynamic shared memory of stage / PST CTAs
    size_t smem_ghost = 0;              // ... of ghost CTAs
    bool preparing = false;             // launch helpers only set kernel attributes
    lssph::Scalars* sc = nullptr;
    lssph::Scalars* sc_host = nullptr;  // pinned copy target for the scalar checks
    int sb = 0, lb = 0;
    cudaGraphExec_t graph[2][lssph::kLists] = {};   // per (state parity, list index)
    int graph_launches = 0;   // kernels per captured step
    int step_sbf = 0;         // state-buffer flip per step (0/1)
    int step_lba = 0;         // list advance per step (mod kLists)
    int64_t launch_counter = 0;
    double last_ms = 0.0;
    int64_t last_launches = 0;
    // per-launch event pairs while profiling (lssph_step_profiled)
    bool profiling = false;
    std::vector<cudaEvent_t> prof_events;
    std::vector<int> prof_kinds;
    size_t prof_next = 0;
    lssph_batch* batch = nullptr;   // the batch this solve is a member of, if any
    lssph::SnapState* snap = nullptr;   // snapshot slots and side stream, set up on first use
    lssph::PPScratch* pp = nullptr;     // lssph_interpolate stream and scratch, set up on first use
    std::string err;
};

namespace lssph {
// Launch a kernel, optionally as a programmatic dependent launch (the kernel may be
// scheduled while the previous kernel in the stream drains; it calls pdl_wait() before
// touching that kernel's results).  Captured into CUDA graphs as programmatic edges.
template <class... KArgs, class... Args>
inline cudaError_t launch_kernel_p(bool pdl, int priority, void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem,
                                   cudaStream_t stream, Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[2];
    unsigned n = 0;
    if (pdl) {
        attr[n].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[n].val.programmaticStreamSerializationAllowed = 1;
        ++n;
    }
    if (priority != 0) {   // scheduling priority of the launch's CTAs (lower value: sooner)
        attr[n].id = cudaLaunchAttributePriority;
        attr[n].val.priority = priority;
        ++n;
    }
    cfg.attrs = n ? attr : nullptr;
    cfg.numAttrs = n;
    return cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

template <class... KArgs, class... Args>
inline cudaError_t launch_kernel(bool pdl, void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem,
                                 cudaStream_t stream, Args&&... args) {
    return launch_kernel_p(pdl, 0, kern, grid, block, smem, stream, std::forward<Args>(args)...);
}

// LSSPH_PDL=0 turns programmatic dependent launches off (default on).
bool pdl_enabled();

// Drop a handle that is being destroyed from the batch that holds it (batch.cu).
void batch_forget(lssph_batch* b, lssph_handle* h);

// Finish and free a handle's asynchronous snapshots (snapshot.cu).
void snapshot_release(lssph_handle* h);
void postproc_release(lssph_handle* h);
// lanes = 0 on a handle not yet measured: measure 2 and 4 lanes now (engine.cu), so that a
// batch member runs the lane count its solo run would.
int resolve_lanes(lssph_handle* h);

// ---- launch plumbing shared by the engine's translation units ----------------------------
inline int blocks_for(long n, int per_block) { return (int)((n + per_block - 1) / per_block); }

// Event pair around one launch while profiling; no-op otherwise (and during capture).
struct ProfScope {
    lssph_handle* h;
    size_t slot = (size_t)-1;
    ProfScope(lssph_handle* hh, int kind) : h(hh) {
        if (!h->profiling) return;
        if (h->prof_next + 2 > h->prof_events.size()) {
            for (int k = 0; k < 64; ++k) {
                cudaEvent_t e;
                if (cudaEventCreate(&e) != cudaSuccess) return;
                h->prof_events.push_back(e);
            }
        }
        slot = h->prof_next;
        h->prof_next += 2;
        h->prof_kinds.push_back(kind);
        cudaEventRecord(h->prof_events[slot], h->stream);
    }
    ~ProfScope() {
        if (slot != (size_t)-1) cudaEventRecord(h->prof_events[slot + 1], h->stream);
    }
};

// Where a launch goes: its tile map (NULL: every tile in order), CTA count, stream, and
// whether it may be a programmatic dependent launch (not right after a fork or join).
struct Where {
    const int* tiles;
    int count;
    cudaStream_t stream;
    bool pdl;
    int priority;   // 0: default
};
inline Where all_tiles(const lssph_handle* h) { return Where{nullptr, h->ntiles, h->stream, h->pdl, 0}; }

// Split shape of the q = 5 LS stage and PST kernels, FP64 or mixed precision
// (split_shape.cu): the pair kernel over the tiles of w, then (after every tile of the
// stage) the solve kernel over all interior particles.
void launch_stage_pairs(lssph_handle* h, const StageCfg& S, const Where& w);
void launch_stage_solve(lssph_handle* h, const StageCfg& S, cudaStream_t stream, bool pdl);
void launch_pst_pairs(lssph_handle* h, const Where& w);
void launch_pst_solve(lssph_handle* h, cudaStream_t stream, bool pdl);
// The handle's kernels can run split: q = 5 LS at 2 or 4 lanes (or lanes = 0).
bool split_capable(const lssph_handle* h);
// A solve of these parameters carries Work::sums: SPH_MODEL 3 at lanes 0, 2 or 4.
inline bool split_sums(const lssph_params& p) {
    return p.sph_model == 3 && (p.lanes == 0 || p.lanes == 2 || p.lanes == 4);
}

// Higher-order LS stage and PST launches, SPH_MODEL 4 / 5 / 6 (highorder.cu).  tiles:
// tile of each CTA (NULL: CTA i runs tile i); while h->preparing they only set the
// kernels' shared-memory attributes.
void launch_stage_hi(lssph_handle* h, const StageCfg& S, const int* tiles, int count, cudaStream_t stream, bool pdl,
                     int priority);
void launch_pst_hi(lssph_handle* h, const int* tiles, int count, cudaStream_t stream, bool pdl, int priority);
}  // namespace lssph
