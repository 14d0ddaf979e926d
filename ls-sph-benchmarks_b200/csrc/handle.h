// handle.h -- the device state of one solve (lssph_handle), shared by the single-solve
// entry points (engine.cu) and the batched time loop (batch.cu).  Internal header.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <utility>
#include <vector>

#include "engine.h"
#include "kernels.cuh"

struct lssph_handle {

    lssph_params p{};
    int num_total = 0, num_int = 0, num_ext = 0;
    int problem = 0;
    bool has_tem = false, p1 = false, pst_on = false;
    int nb_rhs = 4, nb_ghost = 3, nb_pst = 3, wq = 3;
    int G = 4, Gg = 4;
    bool mixed = false;                 // FP32 pair phase, FP64 solve + refinement
    bool pdl = true;                    // programmatic dependent launches in the time step
    bool tuned = false;                 // register budget measured (first solo launch)
    bool tight = false;                 // register budget of stage/PST kernels (autotuned)
    double tune_us[2] = {0.0, 0.0};     // RHS pass time with the loose / tight budget
    lssph::CellGrid grid;
    lssph::VirtualMarkers vm;
    std::vector<int32_t> ptype;
    lssph::Phys P{};
    cudaStream_t stream = nullptr;
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
    std::string err;
};

namespace lssph {
// Launch a kernel, optionally as a programmatic dependent launch (the kernel may be
// scheduled while the previous kernel in the stream drains; it calls pdl_wait() before
// touching that kernel's results).  Captured into CUDA graphs as programmatic edges.
template <class... KArgs, class... Args>
inline cudaError_t launch_kernel(bool pdl, void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem,
                                 cudaStream_t stream, Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = pdl ? attr : nullptr;
    cfg.numAttrs = pdl ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

// LSSPH_PDL=0 turns programmatic dependent launches off (default on).
bool pdl_enabled();

// Drop a handle that is being destroyed from the batch that holds it (batch.cu).
void batch_forget(lssph_batch* b, lssph_handle* h);
}  // namespace lssph
