// batch.cu -- many independent solves advanced by one CUDA graph per time step.
//
// Members are grouped by kind (RHS width, ghost quadrature, RK order, lanes).  A group's
// phase kernel is launched once over the concatenated tiles (or marker chunks) of all
// its members; each CTA finds its solve through a (solve, tile) map and reads that
// solve's descriptor (constants + buffer pointers + buffer parities).  Groups run on
// their own streams, forked from and joined back into the batch stream inside the
// captured step, so small solves of one kind overlap large solves of another.
//
// Parities.  A solo step of problems 2-4 flips the state buffers and advances the cell
// list rotation once per stage and once for PST (RK4: 5 times, RK2: 3); problem 1 flips
// its state buffers once per stage and never scatters.  So after k batch steps a member of
// a group sits at state parity (descriptor's) xor (sbf_g & k) and list index
// (descriptor's) + lba_g k (mod 3), and six graphs (k mod 6) cover every step.
// Descriptors are rewritten whenever the membership changes or a member was advanced on
// its own between batch calls.  The step count lives in device memory: every batched
// kernel derives its parities from it and a last one-thread launch advances it, so one
// graph serves every step.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <string>
#include <tuple>
#include <type_traits>
#include <vector>

#include "handle.h"

using namespace lssph;

namespace {

constexpr int kPeriod = 2 * kLists;   // step period of (state parity, list index)

struct BatchGroup {
    int nb = 4, nbg = 3, wq = 3, rk = 4, G = 4;
    bool p1 = false, pst_on = true, mixed = false, comp = false;
    bool pdl = true;               // programmatic dependent launches between the group's kernels
    const int* tstep = nullptr;    // the batch's device step counter
    int sbf = 1;                   // state-buffer flip per step (0/1)
    int lba = 2;                   // list advance per step (mod kLists)
    std::vector<int> members;      // indices into lssph_batch::members
    SolveDesc* D = nullptr;        // device, one descriptor per member
    int2* tiles = nullptr;         // (solve, tile) per CTA of stage / PST launches
    int2* chunks = nullptr;        // (solve, chunk) per CTA of ghost launches
    int ntiles = 0, nchunks = 0;
    bool tight = false;            // register budget of the stage / PST kernels
    bool split = false;            // mixed precision: pair kernel, then solve kernel (split shape)
    int split_budget = 1;          // budget level of the split shape's pair kernel (1-4)
    int2* blocks = nullptr;        // (solve, block of 128 interior particles) per solve-kernel CTA
    int nblocks = 0;
    int cap_max = 0;               // largest cell slot capacity of the members (pair-kernel smem)
    size_t smem = 0, smem_ghost = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t join = nullptr;
};

}  // namespace

struct lssph_batch {
    std::vector<lssph_handle*> members;
    std::vector<int> base_sb, base_lb;   // member parities the descriptors were written with
    std::vector<int> sbf, lba;           // per member: its group's per-step flip and list advance
    std::vector<BatchGroup> groups;
    bool dirty = true;
    int t = 0;                           // steps since the descriptors were written, mod kPeriod
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, fork = nullptr;
    cudaGraphExec_t graph = nullptr;     // one step of every member (parities from d_t)
    int* d_t = nullptr;                  // device step counter, mod kPeriod
    int graph_launches = 0;
    SolveDesc* all_desc = nullptr;       // device, every member in member order (scalar gather)
    Scalars* d_sc = nullptr;             // device gather buffer: [0, n) before, [n, 2n) after a step call
    Scalars* h_sc = nullptr;             // pinned host copy of it
    size_t sc_cap = 0;
    // the step call in flight (lssph_batch_launch .. lssph_batch_wait)
    bool in_flight = false;
    int flight_steps = 0;
    std::vector<int> sb_start, lb_start;
    double last_ms = 0.0;
    int64_t last_launches = 0;
    std::string err;
};

namespace {

// Tiles per launch above which a group uses the tight register budget even when none of
// its members chose it alone (about two waves at the loose budget's 3 CTAs per SM).
constexpr size_t kTightTiles = 2 * 148 * 3;

int bfail(lssph_batch* b, int code, const std::string& msg) {
    if (b) b->err = msg;
    set_last_error(msg);
    return code;
}

#define BATCH_TRY(b, call)                                                                       \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess)                                                                  \
            return bfail((b), LSSPH_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

template <class F>
void dispatch_lanes(int G, F&& f) {
    switch (G) {
        case 1: f(std::integral_constant<int, 1>{}); break;
        case 2: f(std::integral_constant<int, 2>{}); break;
        case 8: f(std::integral_constant<int, 8>{}); break;
        default: f(std::integral_constant<int, 4>{}); break;
    }
}

template <class K>
void optin(K kernel) {
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tile_smem_bytes(64, 8, true));
}

// Launch (or, with prep, only opt in the shared memory of) one batched phase kernel.
// Precision x lanes: the mixed-precision kernels exist for 2 and 4 lanes.
template <class F>
void dispatch_kind(const BatchGroup& g, F&& f) {
    if (g.mixed && g.comp) {
        if (g.G == 2) f(std::integral_constant<int, 2>{}, std::integral_constant<int, 2>{});
        else f(std::integral_constant<int, 4>{}, std::integral_constant<int, 2>{});
    } else if (g.mixed) {
        if (g.G == 2) f(std::integral_constant<int, 2>{}, std::integral_constant<int, 1>{});
        else f(std::integral_constant<int, 4>{}, std::integral_constant<int, 1>{});
    }
    else dispatch_lanes(g.G, [&](auto GG) { f(GG, std::integral_constant<int, 0>{}); });
}

// Split shape: the pair kernel at the group's budget level (prep: every level), then the
// solve kernel over the group's particle blocks.  MX: 0 FP64, 1 mixed, 2 mixed with
// compensated sums.
template <int NB, bool PST>
void launch_split(const BatchGroup& g, const StageCfg& S, int ps, int pl, bool prep, int* count) {
    constexpr bool TEM = PST ? (NB == 4) : (NB == 5);
    auto run = [&](auto GG, auto MXc) {
        constexpr int G = decltype(GG)::value;
        constexpr int MX = decltype(MXc)::value;
        auto kern_at = [](int t) {
            if constexpr (MX == 0) {
                switch (t) {
                    case 1: return kb_pairs_fp<NB, G, 1, PST>;
                    case 2: return kb_pairs_fp<NB, G, 2, PST>;
                    case 3: return kb_pairs_fp<NB, G, 3, PST>;
                    default: return kb_pairs_fp<NB, G, 4, PST>;
                }
            } else {
                switch (t) {
                    case 1: return kb_pairs_mx<NB, G, 1, MX == 2, PST>;
                    case 2: return kb_pairs_mx<NB, G, 2, MX == 2, PST>;
                    case 3: return kb_pairs_mx<NB, G, 3, MX == 2, PST>;
                    default: return kb_pairs_mx<NB, G, 4, MX == 2, PST>;
                }
            }
        };
        if (prep) {
            for (int t = 1; t <= 4; ++t) optin(kern_at(t));
            return;
        }
        const size_t smem = MX == 0 ? tile_smem_bytes_fpp(g.cap_max, G, TEM) : tile_smem_bytes_mxp(g.cap_max, G, TEM);
        launch_kernel(g.pdl, kern_at(g.split_budget), g.ntiles, PPB * G, smem, g.stream, g.D,
                      BatchMap{g.tiles, g.tstep, g.sbf, g.lba}, ps, pl);
        launch_kernel(g.pdl, kb_solve<NB, PST, (MX == 2)>, g.nblocks, 128, 0, g.stream, g.D,
                      BatchMap{g.blocks, g.tstep, g.sbf, g.lba}, S, ps, pl);
        *count += 2;
    };
    auto lanes = [&](auto MXc) {
        if (g.G == 2) run(std::integral_constant<int, 2>{}, MXc);
        else run(std::integral_constant<int, 4>{}, MXc);
    };
    if (!g.mixed) lanes(std::integral_constant<int, 0>{});
    else if (g.comp) lanes(std::integral_constant<int, 2>{});
    else lanes(std::integral_constant<int, 1>{});
}

void launch_stage(const BatchGroup& g, const StageCfg& S, int ps, int pl, bool prep, int* count) {
    if (g.split) {
        if (g.nb == 1) launch_split<1, false>(g, S, ps, pl, prep, count);
        else if (g.nb == 5) launch_split<5, false>(g, S, ps, pl, prep, count);
        else launch_split<4, false>(g, S, ps, pl, prep, count);
        return;
    }
    dispatch_kind(g, [&](auto GG, auto MXc) {
        constexpr int G = decltype(GG)::value;
        constexpr int MX = decltype(MXc)::value;
        auto run = [&](auto loose, auto tight) {
            if (prep) { optin(loose); optin(tight); return; }
            launch_kernel(g.pdl, g.tight ? tight : loose, g.ntiles, PPB * G, g.smem, g.stream, g.D, BatchMap{g.tiles, g.tstep, g.sbf, g.lba}, S,
                          ps, pl);
            ++*count;
        };
        if (g.nb == 1) run(kb_stage<1, G, false, MX>, kb_stage<1, G, true, MX>);
        else if (g.nb == 5) run(kb_stage<5, G, false, MX>, kb_stage<5, G, true, MX>);
        else run(kb_stage<4, G, false, MX>, kb_stage<4, G, true, MX>);
    });
}

void launch_ghost(const BatchGroup& g, int ps, int pl, int zero_other, int reset_umax, bool prep, int* count) {
    dispatch_lanes(g.G, [&](auto GG) {
        constexpr int G = decltype(GG)::value;
        auto run = [&](auto kern) {
            if (prep) { optin(kern); return; }
            launch_kernel(g.pdl, kern, g.nchunks, PPB * G, g.smem_ghost, g.stream, g.D, BatchMap{g.chunks, g.tstep, g.sbf, g.lba}, ps, pl, zero_other,
                          reset_umax);
            ++*count;
        };
        auto by_wq = [&](auto NBc) {
            constexpr int NB = decltype(NBc)::value;
            if (g.wq == 1) run(kb_ghost<NB, G, 1>);
            else if (g.wq == 6) run(kb_ghost<NB, G, 6>);
            else run(kb_ghost<NB, G, 3>);
        };
        if (g.nbg == 1) by_wq(std::integral_constant<int, 1>{});
        else if (g.nbg == 4) by_wq(std::integral_constant<int, 4>{});
        else by_wq(std::integral_constant<int, 3>{});
    });
}

void launch_pst(const BatchGroup& g, int ps, int pl, bool prep, int* count) {
    if (g.split) {
        const StageCfg S{};
        if (g.nb == 5) launch_split<4, true>(g, S, ps, pl, prep, count);
        else launch_split<3, true>(g, S, ps, pl, prep, count);
        return;
    }
    dispatch_kind(g, [&](auto GG, auto MXc) {
        constexpr int G = decltype(GG)::value;
        constexpr int MX = decltype(MXc)::value;
        auto run = [&](auto loose, auto tight) {
            if (prep) { optin(loose); optin(tight); return; }
            launch_kernel(g.pdl, g.tight ? tight : loose, g.ntiles, PPB * G, g.smem, g.stream, g.D, BatchMap{g.tiles, g.tstep, g.sbf, g.lba}, ps,
                          pl);
            ++*count;
        };
        if (g.nb == 5) run(kb_pst<4, G, false, MX>, kb_pst<4, G, true, MX>);
        else run(kb_pst<3, G, false, MX>, kb_pst<3, G, true, MX>);
    });
}

// One time step of one group, starting at relative parity (ps, pl); the same sequence
// as a solo step (enq_step in engine.cu).
void enq_group_step(const BatchGroup& g, int ps, int pl, bool prep, int* count) {
    const int ns = g.rk == 2 ? 2 : 4;
    for (int s = 1; s <= ns; ++s) {
        StageCfg S{};
        S.mode = MODE_STAGE;
        S.stage = s;
        S.last = (s == ns) ? 1 : 0;
        S.do_scatter = g.p1 ? 0 : 1;
        S.do_umax = g.pst_on ? 1 : 0;
        S.do_steady = g.p1 ? 1 : 0;
        S.write_rhs = 1;
        launch_stage(g, S, ps, pl, prep, count);
        ps ^= 1;
        if (!g.p1) {
            pl = next_list(pl);
            launch_ghost(g, ps, pl, 1, 0, prep, count);
        } else {
            launch_ghost(g, ps, pl, 0, 0, prep, count);
        }
    }
    if (g.pst_on) {
        launch_pst(g, ps, pl, prep, count);
        ps ^= 1;
        pl = next_list(pl);
        launch_ghost(g, ps, pl, 1, 1, prep, count);
    }
    if (g.p1 && !prep) {
        launch_kernel(g.pdl, kb_epilogue, (unsigned)((g.members.size() + 127) / 128), 128, 0, g.stream, g.D,
                      (int)g.members.size());
        ++*count;
    }
}

SolveDesc make_desc(const lssph_handle* h) {
    SolveDesc d;
    std::memset(&d, 0, sizeof(d));
    d.P = h->P;
    d.F[0] = h->F[0];
    d.F[1] = h->F[1];
    for (int l = 0; l < kLists; ++l) d.L[l] = h->L[l];
    d.W = h->W;
    d.V = h->V;
    d.VT = VMTiles{h->vt_tile, h->vt_start, h->vt_vm};
    d.gstart = h->gstart;
    d.glist = h->glist;
    d.sc = h->sc;
    d.ntx = h->ntx;
    d.sb = h->sb;
    d.lb = h->lb;
    d.nchunk = std::max(h->nvt, 1);   // a periodic solve (no ghosts) keeps one bookkeeping CTA
    const double dt = h->p.dt;   // the step sizes enq_stage (engine.cu) hands each stage
    if (h->p.rk == 2) {
        d.dt2[0] = dt / 2.0;
        d.dt2[1] = dt;
    } else {
        d.dt1[0] = dt / 6.0; d.dt2[0] = dt / 2.0;
        d.dt1[1] = dt / 3.0; d.dt2[1] = dt / 2.0;
        d.dt1[2] = dt / 3.0; d.dt2[2] = dt;
        d.dt1[3] = dt / 6.0; d.dt2[3] = 0.0;
    }
    return d;
}

void release_groups(lssph_batch* b) {
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    for (auto& g : b->groups) {
        cudaFree(g.D);
        cudaFree(g.tiles);
        cudaFree(g.chunks);
        cudaFree(g.blocks);
        if (g.join) cudaEventDestroy(g.join);
        if (g.stream) cudaStreamDestroy(g.stream);
    }
    b->groups.clear();
    cudaFree(b->all_desc);
    b->all_desc = nullptr;
}

template <class T>
int upload(lssph_batch* b, T** dst, const std::vector<T>& src) {
    *dst = nullptr;
    BATCH_TRY(b, cudaMalloc(dst, sizeof(T) * std::max<size_t>(src.size(), 1)));
    if (!src.empty()) BATCH_TRY(b, cudaMemcpyAsync(*dst, src.data(), sizeof(T) * src.size(), cudaMemcpyHostToDevice, b->stream));
    return LSSPH_OK;
}

// Regroup the members and rewrite descriptors and CTA maps from their current parities.
int rebuild(lssph_batch* b) {
    BATCH_TRY(b, cudaStreamSynchronize(b->stream));
    release_groups(b);
    const size_t n = b->members.size();
    b->base_sb.assign(n, 0);
    b->base_lb.assign(n, 0);
    b->sbf.assign(n, 0);
    b->lba.assign(n, 0);
    std::map<std::tuple<int, int, int, int, int>, int> index;
    for (size_t i = 0; i < n; ++i) {
        const lssph_handle* h = b->members[i];
        const auto key = std::make_tuple(h->nb_rhs, h->wq, h->p.rk, h->G, h->mixed ? (h->comp ? 2 : 1) : 0);
        auto it = index.find(key);
        if (it == index.end()) {
            BatchGroup g;
            g.nb = h->nb_rhs;
            g.nbg = h->nb_ghost;
            g.wq = h->wq;
            g.rk = h->p.rk;
            g.G = h->G;
            g.mixed = h->mixed;
            g.comp = h->comp;
            g.pdl = pdl_enabled();
            g.p1 = h->p1;
            g.pst_on = h->pst_on;
            const int ns = h->p.rk == 2 ? 2 : 4;
            g.sbf = h->p1 ? (ns & 1) : ((ns + 1) & 1);
            g.lba = h->p1 ? 0 : (ns + 1) % kLists;
            it = index.emplace(key, (int)b->groups.size()).first;
            b->groups.push_back(g);
        }
        b->groups[it->second].members.push_back((int)i);
        b->groups[it->second].tstep = b->d_t;
        b->base_sb[i] = b->members[i]->sb;
        b->base_lb[i] = b->members[i]->lb;
        b->sbf[i] = b->groups[it->second].sbf;
        b->lba[i] = b->groups[it->second].lba;
    }
    std::vector<SolveDesc> all;
    for (auto& g : b->groups) {
        std::vector<SolveDesc> desc;
        std::vector<int2> tiles, chunks, blocks;
        // the split shape needs every member's Work::sums and exists at 2 and 4 lanes
        bool can_split = g.G == 2 || g.G == 4;
        for (size_t s = 0; s < g.members.size(); ++s) can_split = can_split && b->members[g.members[s]]->has_sums;
        for (size_t s = 0; s < g.members.size(); ++s) {
            const lssph_handle* h = b->members[g.members[s]];
            desc.push_back(make_desc(h));
            for (int t = 0; t < h->ntiles; ++t) tiles.push_back(make_int2((int)s, t));
            for (int c = 0; c < std::max(h->nvt, 1); ++c) chunks.push_back(make_int2((int)s, c));
            for (int k = 0; k < (h->num_int + 127) / 128; ++k) blocks.push_back(make_int2((int)s, k));
            g.cap_max = std::max(g.cap_max, h->grid.cap);
            // the split shape (identical results) once any member measured it faster alone
            if (can_split && h->split) {
                g.split = true;
                g.split_budget = std::max(g.split_budget, std::max(h->budget, 1));
            }
            g.smem = std::max(g.smem, h->smem_bytes);
            g.smem_ghost = std::max(g.smem_ghost, h->smem_ghost);
            g.tight = g.tight || h->tight;
        }
        // the tight budget wins once a launch has more tiles than fit at the loose one
        // (3 CTAs per SM); a member that chose it alone keeps it in the group
        g.tight = g.tight || tiles.size() > kTightTiles;
        // mixed precision: a launch past two loose waves is in the throughput regime, where
        // the split shape's occupancy pays (cavity 256^2: 282 vs 317 us per step)
        if (can_split && g.mixed && tiles.size() > kTightTiles) {
            g.split = true;
            g.split_budget = std::max(g.split_budget, 2);
        }
        g.ntiles = (int)tiles.size();
        g.nchunks = (int)chunks.size();
        int rc;
        g.nblocks = (int)blocks.size();
        if ((rc = upload(b, &g.D, desc)) != LSSPH_OK || (rc = upload(b, &g.tiles, tiles)) != LSSPH_OK ||
            (rc = upload(b, &g.chunks, chunks)) != LSSPH_OK || (rc = upload(b, &g.blocks, blocks)) != LSSPH_OK)
            return rc;
        BATCH_TRY(b, cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking));
        BATCH_TRY(b, cudaEventCreateWithFlags(&g.join, cudaEventDisableTiming));
        int unused = 0;
        enq_group_step(g, 0, 0, true, &unused);   // shared-memory opt-in of every kernel used
    }
    for (size_t i = 0; i < n; ++i) all.push_back(make_desc(b->members[i]));
    int rc = upload(b, &b->all_desc, all);
    if (rc != LSSPH_OK) return rc;
    if (b->sc_cap < n) {
        cudaFree(b->d_sc);
        cudaFreeHost(b->h_sc);
        b->d_sc = nullptr;
        b->h_sc = nullptr;
        b->sc_cap = 0;
        BATCH_TRY(b, cudaMalloc(&b->d_sc, 2 * sizeof(Scalars) * n));
        BATCH_TRY(b, cudaMallocHost(&b->h_sc, 2 * sizeof(Scalars) * n));
        b->sc_cap = n;
    }
    BATCH_TRY(b, cudaMemsetAsync(b->d_t, 0, sizeof(int), b->stream));
    BATCH_TRY(b, cudaStreamSynchronize(b->stream));
    b->t = 0;
    b->dirty = false;
    return LSSPH_OK;
}

// Enqueue a read-back of every member's scalars into slot `which` (0: before, 1: after).
int gather_scalars(lssph_batch* b, int which) {
    const int n = (int)b->members.size();
    Scalars* d = b->d_sc + (size_t)which * n;
    kb_gather_scalars<<<(n + 127) / 128, 128, 0, b->stream>>>(b->all_desc, n, d);
    BATCH_TRY(b, cudaGetLastError());
    BATCH_TRY(b, cudaMemcpyAsync(b->h_sc + (size_t)which * n, d, sizeof(Scalars) * n, cudaMemcpyDeviceToHost,
                                 b->stream));
    return LSSPH_OK;
}

int capture(lssph_batch* b, cudaGraphExec_t* out) {
    BATCH_TRY(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    cudaEventRecord(b->fork, b->stream);
    int count = 0;
    for (auto& g : b->groups) {
        cudaStreamWaitEvent(g.stream, b->fork, 0);
        enq_group_step(g, 0, 0, false, &count);
        cudaEventRecord(g.join, g.stream);
        cudaStreamWaitEvent(b->stream, g.join, 0);
    }
    kb_advance<<<1, 1, 0, b->stream>>>(b->d_t);
    ++count;
    cudaGraph_t graph = nullptr;
    BATCH_TRY(b, cudaStreamEndCapture(b->stream, &graph));
    const cudaError_t e = cudaGraphInstantiate(out, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return bfail(b, LSSPH_E_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
    b->graph_launches = count;
    return LSSPH_OK;
}

int member_status(const Scalars& s) {
    if (s.err & ERR_NONFINITE) return LSSPH_E_NONFINITE;
    if (s.err & ERR_OUT_OF_DOMAIN) return LSSPH_E_OUT_OF_DOMAIN;
    if (s.err & ERR_CELL_OVERFLOW) return LSSPH_E_CELL_OVERFLOW;
    return LSSPH_OK;
}

}  // namespace

namespace lssph {
void batch_forget(lssph_batch* b, lssph_handle* h) { lssph_batch_remove(b, h); }
}  // namespace lssph

extern "C" {

int lssph_batch_create(lssph_batch** out) {
    if (!out) return bfail(nullptr, LSSPH_E_BAD_PARAM, "null argument");
    *out = nullptr;
    lssph_batch* b = new lssph_batch();
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&b->ev0) != cudaSuccess || cudaEventCreate(&b->ev1) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaMalloc(&b->d_t, sizeof(int)) != cudaSuccess) {
        lssph_batch_destroy(b);
        return bfail(nullptr, LSSPH_E_CUDA, "stream/event creation failed");
    }
    *out = b;
    return LSSPH_OK;
}

void lssph_batch_destroy(lssph_batch* b) {
    if (!b) return;
    if (b->stream) cudaStreamSynchronize(b->stream);
    for (lssph_handle* h : b->members) h->batch = nullptr;
    release_groups(b);
    cudaFree(b->d_sc);
    cudaFreeHost(b->h_sc);
    cudaFree(b->d_t);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

const char* lssph_batch_error(const lssph_batch* b) { return b ? b->err.c_str() : "null batch"; }

int lssph_batch_add(lssph_batch* b, lssph_handle* h) {
    if (!b || !h) return bfail(b, LSSPH_E_BAD_PARAM, "null argument");
    if (h->batch) return bfail(b, LSSPH_E_BAD_PARAM, "the handle is already a member of a batch");
    if (b->in_flight) return bfail(b, LSSPH_E_BAD_PARAM, "a batch step call is in flight");
    if (h->p.sph_model != 3)
        return bfail(b, LSSPH_E_UNSUPPORTED, "batched solves run the 2nd-order LS-SPH model (SPH_MODEL 3) only");
    // a member with lanes = 0 picks its lane count now, as its first solo launch would
    if (const int rc = resolve_lanes(h)) return bfail(b, rc, "measuring a member's lane count failed");
    b->members.push_back(h);
    h->batch = b;
    b->dirty = true;
    return LSSPH_OK;
}

int lssph_batch_remove(lssph_batch* b, lssph_handle* h) {
    if (!b || !h) return bfail(b, LSSPH_E_BAD_PARAM, "null argument");
    auto it = std::find(b->members.begin(), b->members.end(), h);
    if (it == b->members.end()) return bfail(b, LSSPH_E_BAD_PARAM, "the handle is not a member of this batch");
    if (b->in_flight) {   // a member destroyed mid-call: finish the call first
        b->in_flight = false;
        cudaStreamSynchronize(b->stream);
    }
    cudaStreamSynchronize(b->stream);
    b->members.erase(it);
    h->batch = nullptr;
    b->dirty = true;
    return LSSPH_OK;
}

int lssph_batch_size(const lssph_batch* b) { return b ? (int)b->members.size() : 0; }

int lssph_batch_launch(lssph_batch* b, int32_t nsteps) {
    if (!b) return bfail(nullptr, LSSPH_E_BAD_PARAM, "null batch");
    if (b->in_flight) return bfail(b, LSSPH_E_BAD_PARAM, "a batch step call is already in flight");
    const size_t n = b->members.size();
    b->last_ms = 0.0;
    b->last_launches = 0;
    b->flight_steps = nsteps > 0 ? nsteps : 0;
    if (b->flight_steps == 0 || n == 0) { b->in_flight = true; return LSSPH_OK; }
    // a member stepped on its own since the last batch call: rewrite the descriptors
    for (size_t i = 0; i < n && !b->dirty; ++i) {
        const int sb = b->base_sb[i] ^ (b->sbf[i] & b->t & 1), lb = (b->base_lb[i] + b->lba[i] * b->t) % kLists;
        if (b->members[i]->sb != sb || b->members[i]->lb != lb) b->dirty = true;
    }
    int rc;
    if (b->dirty && (rc = rebuild(b)) != LSSPH_OK) return rc;
    if ((rc = gather_scalars(b, 0)) != LSSPH_OK) return rc;
    b->sb_start.resize(n);
    b->lb_start.resize(n);
    for (size_t i = 0; i < n; ++i) {
        b->sb_start[i] = b->members[i]->sb;
        b->lb_start[i] = b->members[i]->lb;
    }
    BATCH_TRY(b, cudaEventRecord(b->ev0, b->stream));
    for (int st = 0; st < nsteps; ++st) {
        if (!b->graph && (rc = capture(b, &b->graph)) != LSSPH_OK) return rc;
        cudaGraphExec_t ge = b->graph;
        BATCH_TRY(b, cudaGraphLaunch(ge, b->stream));
        b->t = (b->t + 1) % kPeriod;
        for (size_t i = 0; i < n; ++i) {   // members follow the batch's parity
            b->members[i]->sb ^= b->sbf[i];
            b->members[i]->lb = (b->members[i]->lb + b->lba[i]) % kLists;
        }
    }
    BATCH_TRY(b, cudaEventRecord(b->ev1, b->stream));
    if ((rc = gather_scalars(b, 1)) != LSSPH_OK) return rc;
    b->in_flight = true;
    return LSSPH_OK;
}

int lssph_batch_wait(lssph_batch* b, int32_t* status, int32_t* steady, int32_t* steps_taken) {
    if (!b) return bfail(nullptr, LSSPH_E_BAD_PARAM, "null batch");
    if (!b->in_flight) return bfail(b, LSSPH_E_BAD_PARAM, "no batch step call in flight");
    b->in_flight = false;
    const size_t n = b->members.size();
    for (size_t i = 0; i < n; ++i) {
        if (status) status[i] = LSSPH_OK;
        if (steady) steady[i] = 0;
        if (steps_taken) steps_taken[i] = 0;
    }
    const int nsteps = b->flight_steps;
    if (nsteps == 0 || n == 0) return LSSPH_OK;
    BATCH_TRY(b, cudaStreamSynchronize(b->stream));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, b->ev0, b->ev1);
    b->last_ms = ms;
    b->last_launches = (int64_t)nsteps * b->graph_launches;
    const Scalars* s0 = b->h_sc;
    const Scalars* s1v = b->h_sc + n;
    int first = LSSPH_OK;
    for (size_t i = 0; i < n; ++i) {
        const Scalars& s1 = s1v[i];
        const int st = member_status(s1);
        if (status) status[i] = st;
        if (st != LSSPH_OK) {
            b->members[i]->err = lssph_status_string(st);
            if (first == LSSPH_OK) first = st;
        }
        if (steady && s1.steady && !s0[i].steady) steady[i] = s1.steady_step - s0[i].step_count;
        // a member that stopped (steady state, step budget, error) ran the remaining steps
        // as no-ops: its buffers sit where its last executed step left them
        const int executed = s1.step_count - s0[i].step_count;
        if (steps_taken) steps_taken[i] = executed;
        if (executed != nsteps) {
            b->members[i]->sb = b->sb_start[i] ^ (b->sbf[i] & executed & 1);
            b->members[i]->lb = (b->lb_start[i] + b->lba[i] * executed) % kLists;
        }
    }
    if (first != LSSPH_OK) return bfail(b, first, "a batch member stopped with an error (see the status array)");
    return LSSPH_OK;
}

int lssph_batch_step(lssph_batch* b, int32_t nsteps, int32_t* status, int32_t* steady, int32_t* steps_taken) {
    const int rc = lssph_batch_launch(b, nsteps);
    if (rc != LSSPH_OK) return rc;
    return lssph_batch_wait(b, status, steady, steps_taken);
}

int lssph_batch_last_step_stats(const lssph_batch* b, double* device_ms, int64_t* kernel_launches) {
    if (!b) return bfail(nullptr, LSSPH_E_BAD_PARAM, "null batch");
    if (device_ms) *device_ms = b->last_ms;
    if (kernel_launches) *kernel_launches = b->last_launches;
    return LSSPH_OK;
}

}  // extern "C"
