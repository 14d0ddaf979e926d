// mixed_split.cu -- launches of the mixed-precision split shape (kernels.cuh: k_stage_mxp /
// k_stage_mxs, k_pst_mxp / k_pst_mxs): the FP32 pair kernel over a stage's tiles, then the
// FP64 solve-and-update kernel over its interior particles.  The pair kernel has register
// budgets up to 1024 threads per SM, since it holds no FP64 solve; the handle's autotuner
// (engine.cu) times it against the fused mixed kernels and keeps the faster shape.
#include <cuda_runtime.h>

#include "handle.h"

namespace lssph {
namespace {

template <class K>
void optin_mxp(K kernel) {
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tile_smem_bytes(64, 8, true));
}

// Pair kernel at the handle's lanes (2 or 4), budget level (0-4) and sums mode.
template <int NB, bool PST, int G, bool COMP>
void run_mxp(lssph_handle* h, const Where& w) {
    constexpr bool TEM = PST ? (NB == 4) : (NB == 5);
    using K = void (*)(const Phys, const Fld, const Lst, const int*, const int*, const Work, Scalars*, int, const int*);
    auto pick = [](auto T) -> K {
        constexpr int TL = decltype(T)::value;
        if constexpr (PST) return k_pst_mxp<NB, G, TL, COMP>;
        else return k_stage_mxp<NB, G, TL, COMP>;
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
        optin_mxp(kern);
        return;
    }
    const size_t smem = tile_smem_bytes_mxp(h->grid.cap, G, TEM);
    launch_kernel_p(w.pdl, w.priority, kern, w.count, PPB * G, smem, w.stream, h->P, h->F[h->sb], h->L[h->lb],
                    h->gstart, h->glist, h->W, h->sc, h->ntx, w.tiles);
    h->launch_counter++;
}

template <int NB, bool PST>
void dispatch_mxp(lssph_handle* h, const Where& w) {
    if (h->comp) {
        if (h->G == 2) run_mxp<NB, PST, 2, true>(h, w);
        else run_mxp<NB, PST, 4, true>(h, w);
    } else {
        if (h->G == 2) run_mxp<NB, PST, 2, false>(h, w);
        else run_mxp<NB, PST, 4, false>(h, w);
    }
}

// Every budget level of the pair kernels this handle may run (shared-memory opt-in while
// the handle is prepared).
template <int NB, bool PST>
void prepare_mxp(lssph_handle* h, const Where& w) {
    const int b = h->budget, g = h->G;
    for (int G : {2, 4}) {
        h->G = G;
        for (int t = 0; t <= 4; ++t) {
            h->budget = t;
            dispatch_mxp<NB, PST>(h, w);
        }
    }
    h->budget = b;
    h->G = g;
}

}  // namespace

void launch_stage_mxp(lssph_handle* h, const StageCfg&, const Where& w) {
    ProfScope prof(h, LSSPH_KIND_STAGE);
    auto go = [&](auto NBc) {
        constexpr int NB = decltype(NBc)::value;
        if (h->preparing) prepare_mxp<NB, false>(h, w);
        else dispatch_mxp<NB, false>(h, w);
    };
    if (h->nb_rhs == 1) go(std::integral_constant<int, 1>{});
    else if (h->nb_rhs == 5) go(std::integral_constant<int, 5>{});
    else go(std::integral_constant<int, 4>{});
}

void launch_pst_mxp(lssph_handle* h, const Where& w) {
    ProfScope prof(h, LSSPH_KIND_PST);
    if (h->has_tem) {
        if (h->preparing) prepare_mxp<4, true>(h, w);
        else dispatch_mxp<4, true>(h, w);
    } else {
        if (h->preparing) prepare_mxp<3, true>(h, w);
        else dispatch_mxp<3, true>(h, w);
    }
}

void launch_stage_mxs(lssph_handle* h, const StageCfg& S, cudaStream_t stream, bool pdl) {
    if (h->preparing) return;
    ProfScope prof(h, LSSPH_KIND_STAGE);
    const int blocks = blocks_for(h->num_int, 128);
    const Fld& cur = h->F[h->sb];
    const Fld& nxt = h->F[h->sb ^ 1];
    const Lst& Ln = h->L[next_list(h->lb)];
    if (h->nb_rhs == 1) launch_kernel(pdl, k_stage_mxs<1>, blocks, 128, 0, stream, h->P, cur, nxt, Ln, h->gstart, h->W, S, h->sc);
    else if (h->nb_rhs == 5) launch_kernel(pdl, k_stage_mxs<5>, blocks, 128, 0, stream, h->P, cur, nxt, Ln, h->gstart, h->W, S, h->sc);
    else launch_kernel(pdl, k_stage_mxs<4>, blocks, 128, 0, stream, h->P, cur, nxt, Ln, h->gstart, h->W, S, h->sc);
    h->launch_counter++;
}

void launch_pst_mxs(lssph_handle* h, cudaStream_t stream, bool pdl) {
    if (h->preparing) return;
    ProfScope prof(h, LSSPH_KIND_PST);
    const int blocks = blocks_for(h->num_int, 128);
    const Fld& cur = h->F[h->sb];
    const Fld& nxt = h->F[h->sb ^ 1];
    const Lst& Ln = h->L[next_list(h->lb)];
    if (h->has_tem) launch_kernel(pdl, k_pst_mxs<4>, blocks, 128, 0, stream, h->P, cur, nxt, Ln, h->gstart, h->W, h->sc);
    else launch_kernel(pdl, k_pst_mxs<3>, blocks, 128, 0, stream, h->P, cur, nxt, Ln, h->gstart, h->W, h->sc);
    h->launch_counter++;
}

}  // namespace lssph
