// snac_batch.cuh — one launch per kernel type for a whole ensemble of models.
//
// Every model of a batch keeps its own device buffers (the same layout as a
// single-model handle).  A batch adds a table of per-model descriptors
// (mesh, field pointers, configuration) and, for each kind of launch, a list
// of work tiles: (model, block index within that model).  A tile is exactly
// the work one block of the single-model kernel does, so the per-model
// results are the single-model results bit for bit; only the launch
// geometry changes.  A block copies its tile's descriptor to shared memory
// and calls the same kernel body as the single-model kernel.  With a grid
// smaller than the tile list, blocks stride over the list (a persistent
// grid whose size the autotuner chooses).
#pragma once

#include "snac_kernels.cuh"

namespace snac {

struct ModelDesc {
    Mesh m;
    Fields F;
    Config cfg;
    double wave_speed;
};
static_assert(sizeof(ModelDesc) % 8 == 0, "descriptor is copied as 64-bit words");

// per-model status gathered after a batch of steps
struct ModelStatus {
    int status;
    int pad;
    long long err_index;
    long long time_step;
};

// BOP_FUSED: the step's first element launch (models without temperature:
// pending element update + stress update; with temperature: the heat flux,
// the element update waiting for BOP_FUSED_STRESS after the energy hooks)
enum {
    BOP_FUSED = 0,
    BOP_HEAT_FLUX = 1,
    BOP_STRESS = 2,
    BOP_LOOP_NODES = 3,
    BOP_HEAT_NODES = 4,
    BOP_MINLS = 5,
    BOP_FUSED_STRESS = 6
};

__device__ __forceinline__ void load_desc(ModelDesc& dst, const ModelDesc* __restrict__ src) {
    constexpr int W = sizeof(ModelDesc) / 8;
    const long long* s = reinterpret_cast<const long long*>(src);
    long long* d = reinterpret_cast<long long*>(&dst);
    for (int i = threadIdx.x; i < W; i += blockDim.x) d[i] = s[i];
}

// the element bodies for a tile's model: phase 0 from the descriptor (in
// shared memory) when the model has one phase, else the model's phase table
template <int P>
__device__ __forceinline__ void fused_step_any(const ModelDesc& md, int lb, bool count_step = true) {
    if (md.F.mat)
        k_fused_step_body<P, false>(md.m, md.F, md.cfg, lb, count_step);
    else
        k_fused_step_body<P, true>(md.m, md.F, md.cfg, lb, count_step);
}
template <int P>
__device__ __forceinline__ void calc_stresses_any(const ModelDesc& md, int lb) {
    if (md.F.mat)
        k_calc_stresses_body<P, false>(md.m, md.F, md.cfg, lb);
    else
        k_calc_stresses_body<P, true>(md.m, md.F, md.cfg, lb);
}

__device__ __forceinline__ void heat_flux_any(const ModelDesc& md, int lb) {
    if (md.F.mat)
        k_heat_flux_body<false>(md.m, md.F, md.cfg, lb);
    else
        k_heat_flux_body<true>(md.m, md.F, md.cfg, lb);
}
// a temperature model's first launch of a fused step: timeStep++,
// currentTime += dt (once per model), then the heat flux
__device__ __forceinline__ void heat_flux_opening_any(const ModelDesc& md, int lb) {
    if (lb == 0 && threadIdx.x == 0) {
        md.F.sc->time_step += 1;
        md.F.sc->current_time += md.F.sc->dt;
    }
    heat_flux_any(md, lb);
}

// Element-tile kernels: the fused end-of-step/next-stress kernel (or its
// heat variant for models with temperature), the heat flux, the stress update.
template <int OP>
__global__ void __launch_bounds__(ELEM_WARPS * 32, SNAC_ELEM_MINB)
    kb_elements(const ModelDesc* __restrict__ D, const int2* __restrict__ tiles, int ntiles) {
    __shared__ ModelDesc md;
    for (int i = blockIdx.x; i < ntiles; i += gridDim.x) {
        const int2 t = tiles[i];
        __syncthreads();  // the previous tile is done with md
        load_desc(md, D + t.x);
        __syncthreads();
        const int P = md.cfg.constitutive;
        if (OP == BOP_FUSED) {
            if (md.cfg.temperature) {
                heat_flux_opening_any(md, t.y);
            } else {
                switch (P) {
                    case SNAC_RHEOLOGY_ELASTIC: fused_step_any<SNAC_RHEOLOGY_ELASTIC>(md, t.y); break;
                    case SNAC_RHEOLOGY_PLASTIC: fused_step_any<SNAC_RHEOLOGY_PLASTIC>(md, t.y); break;
                    case SNAC_RHEOLOGY_VISCOPLASTIC:
                        fused_step_any<SNAC_RHEOLOGY_VISCOPLASTIC>(md, t.y);
                        break;
                    default: fused_step_any<SNAC_RHEOLOGY_MAXWELL>(md, t.y); break;
                }
            }
        } else if (OP == BOP_FUSED_STRESS) {
            switch (P) {
                case SNAC_RHEOLOGY_ELASTIC: fused_step_any<SNAC_RHEOLOGY_ELASTIC>(md, t.y, false); break;
                case SNAC_RHEOLOGY_PLASTIC: fused_step_any<SNAC_RHEOLOGY_PLASTIC>(md, t.y, false); break;
                case SNAC_RHEOLOGY_VISCOPLASTIC:
                    fused_step_any<SNAC_RHEOLOGY_VISCOPLASTIC>(md, t.y, false);
                    break;
                default: fused_step_any<SNAC_RHEOLOGY_MAXWELL>(md, t.y, false); break;
            }
        } else if (OP == BOP_STRESS) {
            switch (P) {
                case SNAC_RHEOLOGY_ELASTIC: calc_stresses_any<SNAC_RHEOLOGY_ELASTIC>(md, t.y); break;
                case SNAC_RHEOLOGY_PLASTIC: calc_stresses_any<SNAC_RHEOLOGY_PLASTIC>(md, t.y); break;
                case SNAC_RHEOLOGY_VISCOPLASTIC:
                    calc_stresses_any<SNAC_RHEOLOGY_VISCOPLASTIC>(md, t.y);
                    break;
                default: calc_stresses_any<SNAC_RHEOLOGY_MAXWELL>(md, t.y); break;
            }
        } else {
            heat_flux_any(md, t.y);
        }
    }
}

// The same element-tile kernels specialised for one rheology class (plugin,
// temperature on/off): the tile lists are grouped by class, and each class
// present gets its own launch, without the run-time switch (fewer registers).
template <int OP, int P, int TEMP>
__global__ void __launch_bounds__(ELEM_WARPS * 32, SNAC_ELEM_MINB)
    kb_elements_c(const ModelDesc* __restrict__ D, const int2* __restrict__ tiles, int ntiles) {
    __shared__ ModelDesc md;
    for (int i = blockIdx.x; i < ntiles; i += gridDim.x) {
        const int2 t = tiles[i];
        __syncthreads();
        load_desc(md, D + t.x);
        __syncthreads();
        if (OP == BOP_FUSED) {
            if (TEMP)
                heat_flux_opening_any(md, t.y);
            else
                fused_step_any<P>(md, t.y);
        } else if (OP == BOP_FUSED_STRESS) {
            fused_step_any<P>(md, t.y, false);
        } else if (OP == BOP_STRESS) {
            calc_stresses_any<P>(md, t.y);
        } else {
            heat_flux_any(md, t.y);
        }
    }
}

// rheology classes of a batch: index = plugin slot * 2 + temperature
constexpr int NCLASS = 8;
__host__ __device__ constexpr int plugin_slot(int constitutive) {
    return constitutive == SNAC_RHEOLOGY_ELASTIC ? 0 : constitutive == SNAC_RHEOLOGY_PLASTIC ? 1
           : constitutive == SNAC_RHEOLOGY_VISCOPLASTIC                                  ? 2
                                                                                          : 3;
}

// Node-tile kernels (one thread per node, or per element for the minimum
// length scale); the block size is the tile size the tile list was built for.
template <int OP>
__global__ void __launch_bounds__(256) kb_nodes(const ModelDesc* __restrict__ D, const int2* __restrict__ tiles, int ntiles) {
    __shared__ ModelDesc md;
    for (int i = blockIdx.x; i < ntiles; i += gridDim.x) {
        const int2 t = tiles[i];
        __syncthreads();
        load_desc(md, D + t.x);
        __syncthreads();
        if (OP == BOP_LOOP_NODES) {
            const bool vo = md.cfg.vonly != 0;
            switch (md.cfg.dt_type) {
                case SNAC_DT_CONSTANT: k_loop_nodes_body<SNAC_DT_CONSTANT, false>(md.m, md.F, md.cfg, t.y); break;
                case SNAC_DT_DYNAMIC:
                    if (vo) k_loop_nodes_body<SNAC_DT_DYNAMIC, true>(md.m, md.F, md.cfg, t.y);
                    else k_loop_nodes_body<SNAC_DT_DYNAMIC, false>(md.m, md.F, md.cfg, t.y);
                    break;
                default:
                    if (vo) k_loop_nodes_body<SNAC_DT_WAVE, true>(md.m, md.F, md.cfg, t.y);
                    else k_loop_nodes_body<SNAC_DT_WAVE, false>(md.m, md.F, md.cfg, t.y);
                    break;
            }
        } else if (OP == BOP_HEAT_NODES) {
            k_heat_nodes_body(md.m, md.F, md.cfg, t.y);
        } else {
            k_min_length_scale_body(md.m, md.F, t.y);
        }
    }
}

// _Snac_Context_Sync of every model: one thread per model
__global__ void kb_sync(const ModelDesc* __restrict__ D, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) sync_one(D[i].cfg, D[i].F.sc, D[i].wave_speed);
}

// _AbstractContext_Execute_Hook of every model (a step that does not start
// with the fused kernel): timeStep++ and dt = dtFactor * dt
__global__ void kb_begin_step(const ModelDesc* __restrict__ D, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        DevScalars* sc = D[i].F.sc;
        sc->time_step += 1;
        sc->dt = 1.0 * sc->dt;
        sc->current_time += sc->dt;
    }
}

__global__ void kb_status(const ModelDesc* __restrict__ D, int n, ModelStatus* out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const DevScalars* sc = D[i].F.sc;
        out[i].status = sc->status;
        out[i].pad = 0;
        out[i].err_index = sc->err_index;
        out[i].time_step = sc->time_step;
    }
}

}  // namespace snac
