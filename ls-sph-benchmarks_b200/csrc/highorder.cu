// highorder.cu -- launches of the higher-order LS-SPH kernels (SPH_MODEL 4 / 5 / 6) for
// the single-solve engine.  A separate translation unit keeps their instantiations out of
// engine.cu's compile.

#include "handle.h"
#include "kernels_hi.cuh"

namespace lssph {
namespace {

// The attribute is per kernel, shared by every handle: set it for the largest cell
// capacity the engine accepts (64), so a later handle with a smaller capacity cannot
// lower it below what an earlier one launches with.
template <class S, class Kern>
void hi_optin(Kern kern, bool tem) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hi_smem_bytes<S>(64, tem));
}

template <int K, int NB>
void stage_hi(lssph_handle* h, const StageCfg& S, const int* tiles, int count, cudaStream_t stream, bool pdl,
              int priority) {
    if (h->hi_thread) {
        using St = TppShape<K, NB, false>;
        auto kt = k_stage_tpp<K, NB>;
        if (h->preparing) {
            cudaFuncSetAttribute(kt, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tpp_smem_bytes<St>(64, NB == 5));
            return;
        }
        launch_kernel_p(pdl, priority, kt, count, St::NT, tpp_smem_bytes<St>(h->P.cap, NB == 5), stream, h->P,
                        h->F[h->sb], h->F[h->sb ^ 1], h->L[h->lb], h->L[next_list(h->lb)], h->gstart, h->glist, h->W,
                        S, h->sc, h->ntx, tiles);
        h->launch_counter++;
        return;
    }
    using Sh = HiShape<K, NB, false>;
    auto kern = k_stage_hi<K, NB>;
    if (h->preparing) { hi_optin<Sh>(kern, NB == 5); return; }
    launch_kernel_p(pdl, priority, kern, count, 32 * HI_WARPS, hi_smem_bytes<Sh>(h->P.cap, NB == 5), stream, h->P,
                    h->F[h->sb], h->F[h->sb ^ 1], h->L[h->lb], h->L[next_list(h->lb)], h->gstart, h->glist, h->W, S,
                    h->sc, h->ntx, tiles);
    h->launch_counter++;
}

template <int K, int NB>
void pst_hi(lssph_handle* h, const int* tiles, int count, cudaStream_t stream, bool pdl, int priority) {
    if (h->hi_thread) {
        using St = TppShape<K, NB, true>;
        auto kt = k_pst_tpp<K, NB>;
        if (h->preparing) {
            cudaFuncSetAttribute(kt, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tpp_smem_bytes<St>(64, NB == 4));
            return;
        }
        launch_kernel_p(pdl, priority, kt, count, St::NT, tpp_smem_bytes<St>(h->P.cap, NB == 4), stream, h->P,
                        h->F[h->sb], h->F[h->sb ^ 1], h->L[h->lb], h->L[next_list(h->lb)], h->gstart, h->glist, h->W,
                        h->sc, h->ntx, tiles);
        h->launch_counter++;
        return;
    }
    using Sh = HiShape<K, NB, true>;
    auto kern = k_pst_hi<K, NB>;
    if (h->preparing) { hi_optin<Sh>(kern, NB == 4); return; }
    launch_kernel_p(pdl, priority, kern, count, 32 * HI_WARPS, hi_smem_bytes<Sh>(h->P.cap, NB == 4), stream, h->P,
                    h->F[h->sb], h->F[h->sb ^ 1], h->L[h->lb], h->L[next_list(h->lb)], h->gstart, h->glist, h->W,
                    h->sc, h->ntx, tiles);
    h->launch_counter++;
}

template <int NB>
void stage_hi_k(lssph_handle* h, const StageCfg& S, const int* tiles, int count, cudaStream_t stream, bool pdl,
                int priority) {
    if (h->order == 3) stage_hi<3, NB>(h, S, tiles, count, stream, pdl, priority);
    else if (h->order == 4) stage_hi<4, NB>(h, S, tiles, count, stream, pdl, priority);
    else stage_hi<5, NB>(h, S, tiles, count, stream, pdl, priority);
}

template <int NB>
void pst_hi_k(lssph_handle* h, const int* tiles, int count, cudaStream_t stream, bool pdl, int priority) {
    if (h->order == 3) pst_hi<3, NB>(h, tiles, count, stream, pdl, priority);
    else if (h->order == 4) pst_hi<4, NB>(h, tiles, count, stream, pdl, priority);
    else pst_hi<5, NB>(h, tiles, count, stream, pdl, priority);
}

}  // namespace

void launch_stage_hi(lssph_handle* h, const StageCfg& S, const int* tiles, int count, cudaStream_t stream, bool pdl,
                     int priority) {
    if (h->nb_rhs == 1) stage_hi_k<1>(h, S, tiles, count, stream, pdl, priority);
    else if (h->nb_rhs == 5) stage_hi_k<5>(h, S, tiles, count, stream, pdl, priority);
    else stage_hi_k<4>(h, S, tiles, count, stream, pdl, priority);
}

void launch_pst_hi(lssph_handle* h, const int* tiles, int count, cudaStream_t stream, bool pdl, int priority) {
    if (h->has_tem) pst_hi_k<4>(h, tiles, count, stream, pdl, priority);
    else pst_hi_k<3>(h, tiles, count, stream, pdl, priority);
}

}  // namespace lssph
