// split_shape.cu -- launches of the split shape of the q = 5 LS stage and PST kernels
// (kernels.cuh): the pair kernel over a stage's tiles (k_stage_fpp / k_pst_fpp in FP64,
// k_stage_mxp / k_pst_mxp in mixed precision), then the solve-and-update kernel over its
// interior particles (k_stage_solve / k_pst_solve).  The pair kernel holds no LS solve and no
// sums rows in shared memory, so it has register budgets up to 1024 threads per SM; the
// handle's autotuner (engine.cu) times it against the fused kernels and keeps the faster
// shape.  Both shapes give identical results.
#include <cuda_runtime.h>

#include "handle.h"

namespace lssph {
namespace {

template <class K>
void optin_split(K kernel) {
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tile_smem_bytes(64, 8, true));
}

// Pair kernel at the handle's lanes (2 or 4), budget level (0-4) and precision
// (MX: 0 FP64, 1 mixed, 2 mixed with compensated sums).
template <int NB, bool PST, int G, int MX>
void run_pairs(lssph_handle* h, const Where& w) {
    constexpr bool TEM = PST ? (NB == 4) : (NB == 5);
    using K = void (*)(const Phys, const Fld, const Lst, const int*, const int*, const Work, Scalars*, int, const int*);
    auto pick = [](auto T) -> K {
        constexpr int TL = decltype(T)::value;
        if constexpr (MX == 0) {
            if constexpr (PST) return k_pst_fpp<NB, G, TL>;
            else return k_stage_fpp<NB, G, TL>;
        } else {
            if constexpr (PST) return k_pst_mxp<NB, G, TL, MX == 2>;
            else return k_stage_mxp<NB, G, TL, MX == 2>;
        }
    };
    K kern;
    switch (h->budget) {
        case 0: kern = pick(std::integral_constant<int, 0>{}); break;
        case 1: kern = pick(std::integral_constant<int, 1>{}); break;
        case 2: kern = pick(std::integral_constant<int, 2>{}); break;
        case 3: kern = pick(std::integral_constant<int, 3>{}); break;
        default: kern = pick(std::integral_constant<int, 4>{}); break;
    }
    if (h->preparing) {
        optin_split(kern);
        return;
    }
    const size_t smem = MX == 0 ? tile_smem_bytes_fpp(h->grid.cap, G, TEM) : tile_smem_bytes_mxp(h->grid.cap, G, TEM);
    launch_kernel_p(w.pdl, w.priority, kern, w.count, PPB * G, smem, w.stream, h->P, h->F[h->sb], h->L[h->lb],
                    h->gstart, h->glist, h->W, h->sc, h->ntx, w.tiles);
    h->launch_counter++;
}

template <int NB, bool PST>
void dispatch_pairs(lssph_handle* h, const Where& w) {
    if (!h->mixed) {
        if (h->G == 2) run_pairs<NB, PST, 2, 0>(h, w);
        else run_pairs<NB, PST, 4, 0>(h, w);
    } else if (h->comp) {
        if (h->G == 2) run_pairs<NB, PST, 2, 2>(h, w);
        else run_pairs<NB, PST, 4, 2>(h, w);
    } else {
        if (h->G == 2) run_pairs<NB, PST, 2, 1>(h, w);
        else run_pairs<NB, PST, 4, 1>(h, w);
    }
}

// Every lane count and budget level of the pair kernels this handle may run (shared-memory
// opt-in while the handle is prepared).
template <int NB, bool PST>
void prepare_pairs(lssph_handle* h, const Where& w) {
    const int b = h->budget, g = h->G;
    for (int G : {2, 4}) {
        h->G = G;
        for (int t = 0; t <= 4; ++t) {
            h->budget = t;
            dispatch_pairs<NB, PST>(h, w);
        }
    }
    h->budget = b;
    h->G = g;
}

}  // namespace

bool split_capable(const lssph_handle* h) {
    return h->has_sums && !h->classical && h->order == 2 && (h->lanes_auto || h->G == 2 || h->G == 4);
}

void launch_stage_pairs(lssph_handle* h, const StageCfg&, const Where& w) {
    ProfScope prof(h, LSSPH_KIND_STAGE);
    auto go = [&](auto NBc) {
        constexpr int NB = decltype(NBc)::value;
        if (h->preparing) prepare_pairs<NB, false>(h, w);
        else dispatch_pairs<NB, false>(h, w);
    };
    if (h->nb_rhs == 1) go(std::integral_constant<int, 1>{});
    else if (h->nb_rhs == 5) go(std::integral_constant<int, 5>{});
    else go(std::integral_constant<int, 4>{});
}

void launch_pst_pairs(lssph_handle* h, const Where& w) {
    ProfScope prof(h, LSSPH_KIND_PST);
    if (h->has_tem) {
        if (h->preparing) prepare_pairs<4, true>(h, w);
        else dispatch_pairs<4, true>(h, w);
    } else {
        if (h->preparing) prepare_pairs<3, true>(h, w);
        else dispatch_pairs<3, true>(h, w);
    }
}

void launch_stage_solve(lssph_handle* h, const StageCfg& S, cudaStream_t stream, bool pdl) {
    if (h->preparing) return;
    ProfScope prof(h, LSSPH_KIND_STAGE);
    const int blocks = blocks_for(h->num_int, 128);
    const Fld& cur = h->F[h->sb];
    const Fld& nxt = h->F[h->sb ^ 1];
    const Lst& Ln = h->L[next_list(h->lb)];
    auto go = [&](auto kern) {
        launch_kernel(pdl, kern, blocks, 128, 0, stream, h->P, cur, nxt, Ln, h->gstart, h->W, S, h->sc);
    };
    if (h->comp) {   // the compensated mode's solve has one refinement step
        if (h->nb_rhs == 1) go(k_stage_solve<1, true>);
        else if (h->nb_rhs == 5) go(k_stage_solve<5, true>);
        else go(k_stage_solve<4, true>);
    } else {
        if (h->nb_rhs == 1) go(k_stage_solve<1, false>);
        else if (h->nb_rhs == 5) go(k_stage_solve<5, false>);
        else go(k_stage_solve<4, false>);
    }
    h->launch_counter++;
}

void launch_pst_solve(lssph_handle* h, cudaStream_t stream, bool pdl) {
    if (h->preparing) return;
    ProfScope prof(h, LSSPH_KIND_PST);
    const int blocks = blocks_for(h->num_int, 128);
    const Fld& cur = h->F[h->sb];
    const Fld& nxt = h->F[h->sb ^ 1];
    const Lst& Ln = h->L[next_list(h->lb)];
    auto go = [&](auto kern) { launch_kernel(pdl, kern, blocks, 128, 0, stream, h->P, cur, nxt, Ln, h->gstart, h->W, h->sc); };
    if (h->comp) {
        if (h->has_tem) go(k_pst_solve<4, true>);
        else go(k_pst_solve<3, true>);
    } else {
        if (h->has_tem) go(k_pst_solve<4, false>);
        else go(k_pst_solve<3, false>);
    }
    h->launch_counter++;
}

}  // namespace lssph
