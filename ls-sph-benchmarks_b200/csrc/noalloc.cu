// noalloc.cu -- the one entry point of the engine that never allocates device memory.
//
// Who needs it: host codes that cannot call cudaMalloc at the point where they want an
// LS-SPH right-hand side -- for example a solver that has handed all of the GPU's memory
// to its own pool allocator up front, or one that evaluates the RHS from inside a
// time-critical loop where a driver allocation (which may synchronise the device or fail
// under memory pressure) is not acceptable.  Such callers keep the particle state and the
// output arrays in device memory they already own and call lssph_rhs_noalloc.
//
// Everything else the RHS needs (particle volumes, cell keys, the per-cell lists of
// interior and ghost particles, error flags) lives in one statically sized array in
// device memory, g_rhs_scratch below.  The CUDA loader reserves it on every GPU that loads
// this library, for as long as the library stays loaded.
//
// Limits: num_total <= LSSPH_NOALLOC_MAX_PARTICLES, cell grid <= LSSPH_NOALLOC_MAX_CELLS,
// at most LSSPH_NOALLOC_CELL_CAP particles (interior + ghost) per cell.

#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <string>

#include "engine.h"
#include "kernels.cuh"

namespace lssph {
namespace {

using KernelPtr = void (*)(const Phys, const Fld, const Fld, const Lst, const Lst, const int*, const int*, const Work,
                           const StageCfg, Scalars*, int, const int*);

// Byte layout of the scratch array (offsets aligned to 256 bytes).
constexpr size_t align256(size_t n) { return (n + 255) & ~size_t(255); }
constexpr size_t kMaxN = LSSPH_NOALLOC_MAX_PARTICLES;
constexpr size_t kMaxCells = LSSPH_NOALLOC_MAX_CELLS;
constexpr int kCap = LSSPH_NOALLOC_CELL_CAP;
constexpr size_t kOffVol = 0;                                                  // double[kMaxN]
constexpr size_t kOffKey = align256(kOffVol + sizeof(double) * kMaxN);          // int[kMaxN]
constexpr size_t kOffCnt = align256(kOffKey + sizeof(int) * kMaxN);            // int[kMaxCells]
constexpr size_t kOffGcnt = align256(kOffCnt + sizeof(int) * kMaxCells);       // int[kMaxCells]
constexpr size_t kOffGstart = align256(kOffGcnt + sizeof(int) * kMaxCells);    // int[kMaxCells + 1]
constexpr size_t kOffGlist = align256(kOffGstart + sizeof(int) * (kMaxCells + 1));  // int[kMaxN]
constexpr size_t kOffSlots = align256(kOffGlist + sizeof(int) * kMaxN);        // int[kMaxCells * kCap]
constexpr size_t kOffScalars = align256(kOffSlots + sizeof(int) * kMaxCells * kCap);
constexpr size_t kScratchBytes = align256(kOffScalars + sizeof(Scalars));

// The scratch.  Host code must not use this name as a device address: it obtains the
// device address with cudaGetSymbolAddress (scratch_base below).
static __device__ __align__(256) unsigned char g_rhs_scratch[kScratchBytes];

// ---- set-up kernels -------------------------------------------------------------------
// Volumes of all particles, cell keys (ghosts: division form of init_cell_mod.f90:76-78;
// interior: multiplication form of update_cell_mod.f90:53-55), per-cell ghost counts and
// the scatter of interior particles into their cells.
__global__ void k_na_keys(const Phys P, double h_eff, const Fld F, Lst L, int* gkey, int* gcnt, Scalars* sc) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.num_total) return;
    F.vol[i] = P.SP_mass / F.rho[i];
    if (i < P.num_int) {
        const int k = cell_key_mul(P, F.x[i], F.y[i], sc);
        gkey[i] = k;
        if (k < 0) return;
        const int pos = atomicAdd(L.cnt + k, 1);
        if (pos < P.cap) L.slots[(size_t)k * P.cap + pos] = i;
        else atomicOr(&sc->err, ERR_CELL_OVERFLOW);
    } else {
        const double cxd = ceil(F.x[i] / h_eff), cyd = ceil(F.y[i] / h_eff);
        if (!(cxd >= 1.0 && cxd <= (double)P.nx && cyd >= 1.0 && cyd <= (double)P.ny)) {
            atomicOr(&sc->err, ERR_OUT_OF_DOMAIN);
            gkey[i] = -1;
            return;
        }
        const int k = ((int)cxd - 1) + ((int)cyd - 1) * P.nx;
        gkey[i] = k;
        atomicAdd(gcnt + k, 1);
    }
}

// Exclusive scan of the ghost counts (one CTA of 1024 threads).
__global__ void k_na_scan(int ncell, const int* gcnt, int* gstart) {
    __shared__ int part[1024];
    const int t = threadIdx.x, per = (ncell + 1023) / 1024;
    const int b = t * per, e = min(ncell, b + per);
    int s = 0;
    for (int c = b; c < e; ++c) s += gcnt[c];
    part[t] = s;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
        const int v = t >= off ? part[t - off] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    int run = part[t] - s;
    for (int c = b; c < e; ++c) { gstart[c] = run; run += gcnt[c]; }
    if (t == 1023) gstart[ncell] = part[1023];
}

// Ghost lists per cell in ascending particle index (the static list of
// init_cell_mod.f90:105-109): ghosts are placed with a per-cell cursor, then each cell
// sorts its few entries.
__global__ void k_na_ghosts(const Phys P, const int* gkey, const int* gstart, int* gcursor, int* glist) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= P.num_ext) return;
    const int i = P.num_int + g;
    const int k = gkey[i];
    if (k < 0) return;
    const int pos = atomicAdd(gcursor + k, 1);
    glist[gstart[k] + pos] = i;
}

__global__ void k_na_sort_ghosts(const Phys P, const int* cnt, const int* gstart, int* glist, Scalars* sc) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.ncell) return;
    const int b = gstart[c], n = gstart[c + 1] - b;
    if (cnt[c] + n > P.cap) atomicOr(&sc->err, ERR_CELL_OVERFLOW);   // interior + ghosts per cell
    for (int k = 1; k < n; ++k) {
        const int v = glist[b + k];
        int t = k;
        while (t > 0 && glist[b + t - 1] > v) { glist[b + t] = glist[b + t - 1]; --t; }
        glist[b + t] = v;
    }
}

// ---- host side ----------------------------------------------------------------------------
// The tile kernels this entry point launches, by lanes per particle.
template <int NB>
KernelPtr stage_kernel(int lanes) {
    switch (lanes) {
        case 1: return k_stage<NB, 1>;
        case 2: return k_stage<NB, 2>;
        default: return k_stage<NB, 4>;
    }
}

// With the caller's device current: the device address of the scratch array, and the
// shared-memory opt-in of the kernel about to run.  Both are looked up on every call (they
// allocate nothing), so nothing goes stale when the caller resets the device or switches
// contexts between calls.
template <int NB>
int scratch_base(int lanes, unsigned char** out, std::string* msg) {
    void* ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_rhs_scratch);
    if (e != cudaSuccess) { *msg = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e); return LSSPH_E_CUDA; }
    const int bytes = (int)tile_smem_bytes(kCap, lanes, NB == 5);
    const cudaError_t a = cudaFuncSetAttribute(stage_kernel<NB>(lanes), cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (a != cudaSuccess) { *msg = std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(a); return LSSPH_E_CUDA; }
    *out = static_cast<unsigned char*>(ptr);
    return LSSPH_OK;
}

}  // namespace
}  // namespace lssph

using namespace lssph;

extern "C" int lssph_rhs_noalloc(const lssph_params* pin, int32_t num_total, int32_t num_int, const double* x,
                                 const double* y, const double* u, const double* v, const double* rho,
                                 const double* pre, const double* tem, double* rhs_u, double* rhs_v, double* rhs_rho,
                                 double* rhs_tem, void* stream) {
    std::string msg;
    auto fail = [&](int code, const std::string& m) { set_last_error(m); return code; };
    if (!pin || !x || !y || !u || !v || !rho || !pre || !rhs_u || !rhs_v || !rhs_rho)
        return fail(LSSPH_E_BAD_PARAM, "lssph_rhs_noalloc: null argument");
    if (check_param(pin, &msg) != LSSPH_OK) return fail(LSSPH_E_BAD_PARAM, msg);
    lssph_params p = *pin;
    init_param(&p);
    if (p.target_problem == 1 || p.sph_model != 3 || p.precision != LSSPH_PRECISION_FP64)
        return fail(LSSPH_E_UNSUPPORTED, "lssph_rhs_noalloc: FP64 SPH_MODEL 3 for problems 2-4 only");
    if (p.periodic)
        return fail(LSSPH_E_UNSUPPORTED, "lssph_rhs_noalloc: the closed box only (its cell grid has no periodic wrap)");
    if (!(p.lanes == 0 || p.lanes == 1 || p.lanes == 2 || p.lanes == 4))
        return fail(LSSPH_E_UNSUPPORTED, "lssph_rhs_noalloc: lanes must be 1, 2 or 4 (0 means 4)");
    const int lanes = p.lanes == 0 ? 4 : p.lanes;
    if (p.target_problem == 4 && (!tem || !rhs_tem)) return fail(LSSPH_E_BAD_PARAM, "lssph_rhs_noalloc: tem required");
    const int nx = (int)std::ceil((p.len_x + 2.0 * p.WL_thick) / p.h_eff);
    const int ny = (int)std::ceil((p.len_y + 2.0 * p.WL_thick) / p.h_eff);
    if (num_int <= 0 || num_total <= num_int) return fail(LSSPH_E_BAD_PARAM, "lssph_rhs_noalloc: bad particle counts");
    if ((size_t)num_total > kMaxN || (size_t)nx * ny > kMaxCells)
        return fail(LSSPH_E_CAPACITY, "lssph_rhs_noalloc: at most " + std::to_string(kMaxN) + " particles and " +
                                          std::to_string(kMaxCells) + " cells (got " + std::to_string(num_total) +
                                          " particles, " + std::to_string((long)nx * ny) + " cells)");
    unsigned char* base = nullptr;
    const int rc = p.target_problem == 4 ? scratch_base<5>(lanes, &base, &msg) : scratch_base<4>(lanes, &base, &msg);
    if (rc != LSSPH_OK) return fail(rc, "lssph_rhs_noalloc: " + msg);
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    Phys P{};
    P.problem = p.target_problem; P.kt = p.kernel_type; P.rk = p.rk; P.wall_model = p.wall_model;
    P.nx = nx; P.ny = ny; P.ncell = nx * ny; P.cap = kCap;
    P.num_total = num_total; P.num_int = num_int; P.num_ext = num_total - num_int;
    P.h = p.h; P.ih1 = 1.0 / p.h; P.ih2A = P.ih1 / p.h; P.ih2B = P.ih1 * P.ih1;
    P.h_eff_sq = p.h_eff * p.h_eff; P.inv_h_eff = 1.0 / p.h_eff; P.SP_mass = p.SP_mass; P.W_ave = p.W_ave;
    P.wnorm = kernel_norm(p.kernel_type, p.h); P.dt = p.dt;
    P.c_sq = p.sound_speed * p.sound_speed; P.rho_ref = p.rho_ref; P.vis_ref = p.vis_ref;
    P.delta = ((p.coe_delta_sph * p.sound_speed) * p.h) * p.zeta_RSST;
    P.zeta_sq = p.zeta_RSST * p.zeta_RSST; P.xi_sq = p.xi_VIM * p.xi_VIM;
    P.alpha_ref = p.alpha_ref; P.gravity = p.gravity; P.tem_ave = p.tem_ave; P.thermal_dif = p.thermal_dif;
    P.iWave = 1.0 / p.W_ave; P.izeta2 = 1.0 / (p.zeta_RSST * p.zeta_RSST); P.ixi2 = 1.0 / (p.xi_VIM * p.xi_VIM);
    P.m3h = -3.0 / p.h; P.m5h = -5.0 / p.h;

    Fld F{};
    F.x = const_cast<double*>(x); F.y = const_cast<double*>(y); F.u = const_cast<double*>(u);
    F.v = const_cast<double*>(v); F.rho = const_cast<double*>(rho); F.pre = const_cast<double*>(pre);
    F.tem = const_cast<double*>(tem);
    F.vol = reinterpret_cast<double*>(base + kOffVol);
    int* key = reinterpret_cast<int*>(base + kOffKey);
    Lst L{reinterpret_cast<int*>(base + kOffCnt), reinterpret_cast<int*>(base + kOffSlots)};
    int* gcnt = reinterpret_cast<int*>(base + kOffGcnt);
    int* gstart = reinterpret_cast<int*>(base + kOffGstart);
    int* glist = reinterpret_cast<int*>(base + kOffGlist);
    Scalars* sc = reinterpret_cast<Scalars*>(base + kOffScalars);
    Work W{};
    W.rhs_u = rhs_u; W.rhs_v = rhs_v; W.rhs_rho = rhs_rho; W.rhs_tem = rhs_tem; W.key = key;

    // The scratch keeps the previous call's contents: clear the counters and flags.
    const size_t nc = (size_t)P.ncell;
    cudaError_t e = cudaMemsetAsync(L.cnt, 0, sizeof(int) * nc, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(gcnt, 0, sizeof(int) * nc, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(sc, 0, sizeof(Scalars), s);
    if (e != cudaSuccess) return fail(LSSPH_E_CUDA, std::string("lssph_rhs_noalloc: ") + cudaGetErrorString(e));
    k_na_keys<<<(num_total + 255) / 256, 256, 0, s>>>(P, p.h_eff, F, L, key, gcnt, sc);
    k_na_scan<<<1, 1024, 0, s>>>(P.ncell, gcnt, gstart);
    e = cudaMemsetAsync(gcnt, 0, sizeof(int) * nc, s);   // reused as the ghost cursor
    if (e != cudaSuccess) return fail(LSSPH_E_CUDA, std::string("lssph_rhs_noalloc: ") + cudaGetErrorString(e));
    k_na_ghosts<<<(P.num_ext + 255) / 256, 256, 0, s>>>(P, key, gstart, gcnt, glist);
    k_na_sort_ghosts<<<(P.ncell + 255) / 256, 256, 0, s>>>(P, L.cnt, gstart, glist, sc);

    StageCfg S{};
    S.mode = MODE_RHS_ONLY;
    S.stage = 1;
    S.write_rhs = 1;
    const int ntx = (nx + TX - 1) / TX, nty = (ny + TY - 1) / TY;
    const size_t sm = tile_smem_bytes(kCap, lanes, p.target_problem == 4);
    if (p.target_problem == 4)
        stage_kernel<5>(lanes)<<<ntx * nty, PPB * lanes, sm, s>>>(P, F, F, L, L, gstart, glist, W, S, sc, ntx, nullptr);
    else
        stage_kernel<4>(lanes)<<<ntx * nty, PPB * lanes, sm, s>>>(P, F, F, L, L, gstart, glist, W, S, sc, ntx, nullptr);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(LSSPH_E_CUDA, std::string("lssph_rhs_noalloc: launch: ") + cudaGetErrorString(e));
    Scalars hs{};
    e = cudaMemcpyAsync(&hs, sc, sizeof(Scalars), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(LSSPH_E_CUDA, std::string("lssph_rhs_noalloc: ") + cudaGetErrorString(e));
    if (hs.err & ERR_OUT_OF_DOMAIN) return fail(LSSPH_E_OUT_OF_DOMAIN, "lssph_rhs_noalloc: a particle is outside the cell grid");
    if (hs.err & ERR_CELL_OVERFLOW)
        return fail(LSSPH_E_CELL_OVERFLOW, "lssph_rhs_noalloc: more than " + std::to_string(kCap) + " particles in a cell");
    return LSSPH_OK;
}
