// snac_api.cu — host side of the C ABI declared in include/snac_gpu.h.
//
// A handle owns the device state of one model, one CUDA stream and two CUDA
// graphs (one step each, for the two coordinate-buffer parities).  The
// initial conditions that the reference applies on the host before
// SnacTimeStepZero are computed here too (velocity BCs, the temperature
// sweep, the hydrostatic column integration, the plugin dt bounds).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "snac_gpu.h"
#include "snac_adjoint.cuh"
#include "snac_batch.cuh"
#include "snac_output.cuh"
#include "snac_slab_plan.h"
#include "snac_kernels.cuh"

using namespace snac;

// Dump / checkpoint files in the reference's format (see snac_gpu_output_open)
struct OutputState {
    enum {
        D_SR, D_ST, D_HP, D_PH, D_CO, D_VE, D_FO, D_TEN, D_PL, D_VI, D_TE,
        C_PH, C_CO, C_VE, C_TEN, C_PL, C_VI, C_TE, T_STEP, T_CP, T_SIM, NF
    };
    std::string dir;
    unsigned rank = 0, dump_every = 1, checkpoint_every = 0, max_steps = 0;
    FILE* f[NF] = {};
    char* dstage = nullptr;   // device staging
    char* pinned = nullptr;   // pinned host copy
    size_t cap = 0;
    cudaEvent_t ready = nullptr;
    std::thread writer;
    struct Piece {
        int file;
        size_t off, bytes;
    };
    std::vector<Piece> pieces;
    std::string lines[2];     // timeStep / checkpointTimeStep records of the pending write
    size_t scal_off = 0;      // where the step scalars sit in the pinned copy
    bool dump = false, cp = false;
    int err = 0;
    int want = 0;             // the last element-scalar request sent to the device
};

// Streams, events and node staging of snac_gpu_step_host (created on its
// first call): uploads run on `in`, downloads on `out`, kernels on the
// handle's stream, ordered slab by slab through the events.
constexpr int STEP_HOST_MAX_CHUNKS = 64;
struct HostStep {
    cudaStream_t in = nullptr, out = nullptr;
    cudaEvent_t start = nullptr, done = nullptr, nodes_in = nullptr, nodes_rest = nullptr;
    cudaEvent_t ev_in[STEP_HOST_MAX_CHUNKS] = {}, ev_elems[STEP_HOST_MAX_CHUNKS] = {};
    double* stage_in = nullptr;   // [nn][3] coordinates, [nn][3] velocities, [nn] temperatures, as the host holds them
    double* stage_out = nullptr;  // the same rows
    bool ready = false;
};

struct snac_gpu {
    Mesh mesh{};
    Config cfg{};
    int constitutive = 0;
    int temperature = 0;
    int has_density = 0;
    int n_phases = 0;
    double wave_speed = 0.0;
    cudaStream_t stream = nullptr;
    bool own_stream = true;  // false for the models of a batch, which share the batch's stream
    long long alloc_bytes = 0;  // device bytes allocated for this handle since creation (snac_gpu_device_bytes)
    // device buffers
    double4* pos[2] = {nullptr, nullptr};
    double4* vel = nullptr;
    double4* force = nullptr;
    double* stress = nullptr;
    double* eps_p = nullptr;
    double* pst = nullptr;   // plastic strain tensor [nq][6] (visco-plastic with a Drucker-Prager phase)
    int dp = 0;              // the visco-plastic model has a Drucker-Prager phase: SNAC_VP_DP kernel instances
    int abi = SNAC_GPU_ABI_VERSION;  // version of the descriptor it was created from (state-view size)
    double* visc = nullptr;
    double* density = nullptr;
    double* vol = nullptr;
    double* hflux = nullptr;
    double* tpre = nullptr;
    double* fterm = nullptr;
    double* fgrav = nullptr;
    double* fmass = nullptr;
    uchar4* bc = nullptr;
    double* vbc_val = nullptr;
    double* tbc_val = nullptr;
    unsigned char* mat = nullptr;
    DevMaterial* mats = nullptr;
    double* coh_scale = nullptr;
    double* fric_scale = nullptr;
    double* visc_scale = nullptr;
    DevScalars* sc = nullptr;
    double* stage = nullptr;  // host-transfer staging, 3 doubles per node (first upload/download)
    double* escal = nullptr;  // [ne][4] element scalars for the dump files (allocated by snac_gpu_output_open)
    double* residual_fr = nullptr;  // [nn] Winkler residual force
    double* topo_scratch = nullptr;  // [nnx * nnz] topography-diffusion scratch
    OutputState* out = nullptr;
    HostStep* hs = nullptr;  // snac_gpu_step_host's streams and staging
    // host mirror of the step bookkeeping
    int parity = 0;
    long long time_step = 0;
    bool zero_done = false;
    cudaGraphExec_t graph[2][2][2] = {};  // [heat flux formed][fused][parity]
    bool pending = false;  // the element update of the last step is deferred into the next kernel
    // temperature runs: the heat flux of the next step was formed at the end
    // of the last graph step (k_heat_flux_min_length_scale); anything
    // else that runs or changes the state clears it
    bool hflux_ready = false;
    // kernel-by-kernel timing (snac_gpu_profile_step)
    snac_kernel_time* prof = nullptr;
    int prof_n = 0, prof_max = 0;
    cudaEvent_t prof_ev[64];
    long long launches = 0;
    int steps_kernels[2][2] = {};  // kernels of a step graph [heat flux formed][fused]
    char err[512] = {0};
    long long err_index = -1;
};

namespace {

int set_err(snac_gpu* h, int code, long long idx, const char* fmt, ...) {
    if (!h) return code;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(h->err, sizeof h->err, fmt, ap);
    va_end(ap);
    h->err_index = idx;
    return code;
}

#define CK(call)                                                                                     \
    do {                                                                                             \
        cudaError_t e_ = (call);                                                                     \
        if (e_ != cudaSuccess) return set_err(h, SNAC_GPU_ECUDA, -1, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

template <class T>
int dalloc(snac_gpu* h, T** p, size_t n) {
    if (n == 0) n = 1;
    cudaError_t e = cudaMalloc((void**)p, n * sizeof(T));
    if (e != cudaSuccess) return set_err(h, SNAC_GPU_ENOMEM, -1, "cudaMalloc(%zu bytes): %s", n * sizeof(T), cudaGetErrorString(e));
    h->alloc_bytes += (long long)(n * sizeof(T));
    e = cudaMemsetAsync(*p, 0, n * sizeof(T), h->stream);
    if (e != cudaSuccess) return set_err(h, SNAC_GPU_ECUDA, -1, "cudaMemset: %s", cudaGetErrorString(e));
    return 0;
}

bool wall_has(int wall, int i, int j, int k, int nnx, int nny, int nnz) {
    switch (wall) {
        case SNAC_WALL_BACK: return k == 0;
        case SNAC_WALL_LEFT: return i == 0;
        case SNAC_WALL_BOTTOM: return j == 0;
        case SNAC_WALL_RIGHT: return i == nnx - 1;
        case SNAC_WALL_TOP: return j == nny - 1;
        case SNAC_WALL_FRONT: return k == nnz - 1;
        case SNAC_WALL_ALL: return true;
        default: return false;
    }
}

// Host copy of a phase for the device.  Angles that are constant over the
// whole softening table get their sin/tan from the host C library.
DevMaterial to_dev(const snac_material& s, bool fric_scaled, int dp_maxit, double dp_tol) {
    DevMaterial d;
    memset(&d, 0, sizeof d);
    d.density = s.density;
    d.alpha = s.alpha;
    d.beta = s.beta;
    d.lambda = s.lambda;
    d.mu = s.mu;
    d.nsegments = s.nsegments;
    d.yield_mc = s.yield_mohr_coulomb;
    for (int i = 0; i <= SNAC_MAX_SEGMENTS; i++) {
        d.plstrain[i] = s.plstrain[i];
        d.fric[i] = s.friction_angle[i];
        d.dil[i] = s.dilation_angle[i];
        d.coh[i] = s.cohesion[i];
    }
    d.ten_off = s.ten_off;
    d.vis_min = s.vis_min;
    d.vis_max = s.vis_max;
    d.refvisc = s.refvisc;
    d.refsrate = s.refsrate;
    d.reftemp = s.reftemp;
    d.H = s.activation_e;
    d.srexponent = s.srexponent;
    d.thermal_conduct = s.thermal_conduct;
    d.heat_capacity = s.heat_capacity;
    d.vp_expo = (1. / s.srexponent) - 1.;
    d.vp_hr = s.activation_e / 8.31448;
    d.vp_irt = 1. / (s.reftemp + 273.15);
    d.vp_zrs = 1. / s.refsrate;
    const double degrad = 3.14159265358979323846 / 180.0f;
    bool fc = !fric_scaled, dc = true;
    for (int i = 1; i <= s.nsegments; i++) {
        if (s.friction_angle[i] != s.friction_angle[0]) fc = false;
        if (s.dilation_angle[i] != s.dilation_angle[0]) dc = false;
    }
    d.fric_const = fc;
    d.dil_const = dc;
    d.fric0 = s.friction_angle[0];
    d.sin_fric0 = sin(d.fric0 * degrad);
    d.tan_fric0 = tan(d.fric0 * degrad);
    d.dil0 = s.dilation_angle[0];
    d.sin_dil0 = sin(d.dil0 * degrad);
    d.tan_dil0 = tan(d.dil0 * degrad);
    d.dp_maxit = dp_maxit;
    d.dp_tol = dp_tol;
    d.anphi0 = (1.0f + d.sin_fric0) / (1.0f - d.sin_fric0);
    d.anpsi0 = (1.0f + d.sin_dil0) / (1.0f - d.sin_dil0);
    d.sq_anphi0 = sqrt(d.anphi0);
    d.ztan_fric0 = 1.0 / d.tan_fric0;
    for (int i = 0; i < SNAC_MAX_SEGMENTS; i++)
        d.zpl[i] = i < s.nsegments ? 1.0 / (s.plstrain[i + 1] - s.plstrain[i]) : 0.0;
    return d;
}

Fields fields_at(const snac_gpu* h, int parity) {
    Fields F;
    F.pos = h->pos[parity];
    F.pos_next = h->pos[parity ^ 1];
    F.vel = h->vel;
    F.force = h->force;
    F.stress = h->stress;
    F.eps_p = h->eps_p;
    F.pst = h->pst;
    F.visc = h->visc;
    F.density = h->density;
    F.vol = h->vol;
    F.hflux = h->hflux;
    F.tpre = h->tpre;
    F.fterm = h->fterm;
    F.fgrav = h->fgrav;
    F.fmass = h->fmass;
    F.bc = h->bc;
    F.vbc_val = h->vbc_val;
    F.tbc_val = h->tbc_val;
    F.mat = h->mat;
    F.mats = h->mats;
    F.escal = h->escal;
    F.residual_fr = h->residual_fr;
    F.coh_scale = h->coh_scale;
    F.fric_scale = h->fric_scale;
    F.visc_scale = h->visc_scale;
    F.sc = h->sc;
    return F;
}

Fields fields(const snac_gpu* h) { return fields_at(h, h->parity); }

unsigned elem_blocks(const Mesh& m) { return (unsigned)((m.ne + ELEM_PER_BLOCK - 1) / ELEM_PER_BLOCK); }
unsigned node_blocks(const Mesh& m) { return (unsigned)((m.nn + 127) / 128); }

// called right after each launch: checks it and, when profiling, records an
// event behind it (the event before the first launch is recorded by the caller)
int launch_check_named(snac_gpu* h, const char* name) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_err(h, SNAC_GPU_ECUDA, -1, "kernel launch: %s", cudaGetErrorString(e));
    if (h->prof && h->prof_n < h->prof_max && h->prof_n < 63) {
        cudaEventRecord(h->prof_ev[h->prof_n + 1], h->stream);
        snprintf(h->prof[h->prof_n].name, sizeof h->prof[h->prof_n].name, "%s", name);
        h->prof_n++;
    }
    return 0;
}
#define launch_check(h) launch_check_named((h), __func__)

// the topography hooks do something when diffusion is on, or when a
// non-positive criterion lets the edge copy run with topoGradMax = 0
bool topo_on(const Config& c) { return c.topo_kappa > 0 || !(c.topo_crit > 0); }

template <int P>
void launch_stress(snac_gpu* h, const Fields& F, const Config& c) {
    if (h->mat)
        k_calc_stresses<P, false><<<elem_blocks(h->mesh), ELEM_WARPS * 32, 0, h->stream>>>(h->mesh, F, c);
    else
        k_calc_stresses<P, true><<<elem_blocks(h->mesh), ELEM_WARPS * 32, 0, h->stream>>>(h->mesh, F, c);
}
template <int P>
void launch_update(snac_gpu* h, const Fields& F, const Config& c, int pending) {
    k_update_elements<P><<<elem_blocks(h->mesh), ELEM_WARPS * 32, 0, h->stream>>>(h->mesh, F, c, pending);
}
template <int P>
void launch_fused(snac_gpu* h, const Fields& F, const Config& c) {
    if (h->mat)
        k_fused_step<P, false><<<elem_blocks(h->mesh), ELEM_WARPS * 32, 0, h->stream>>>(h->mesh, F, c);
    else
        k_fused_step<P, true><<<elem_blocks(h->mesh), ELEM_WARPS * 32, 0, h->stream>>>(h->mesh, F, c);
}
// count_step: this launch opens the step (timeStep++, currentTime += dt)
int op_energy_elements(snac_gpu* h, int count_step = 0) {
    if (!h->temperature) return 0;
    if (h->mat)
        k_heat_flux<false><<<elem_blocks(h->mesh), ELEM_WARPS * 32, 0, h->stream>>>(h->mesh, fields(h), h->cfg,
                                                                                   count_step);
    else
        k_heat_flux<true><<<elem_blocks(h->mesh), ELEM_WARPS * 32, 0, h->stream>>>(h->mesh, fields(h), h->cfg,
                                                                                  count_step);
    h->launches++;
    if (count_step) h->time_step++;
    return launch_check_named(h, "k_heat_flux");
}

template <int P>
void launch_fused_stress(snac_gpu* h, const Fields& F, const Config& c) {
    if (h->mat)
        k_fused_stress<P, false><<<elem_blocks(h->mesh), ELEM_WARPS * 32, 0, h->stream>>>(h->mesh, F, c);
    else
        k_fused_stress<P, true><<<elem_blocks(h->mesh), ELEM_WARPS * 32, 0, h->stream>>>(h->mesh, F, c);
}

// temperature runs: the pending element update of the previous step with
// this step's stress update, after the energy hooks
int op_fused_stress(snac_gpu* h) {
    Fields F = fields(h);
    Config c = h->cfg;
    c.time_step_zero = 0;
    switch (h->constitutive) {
        case SNAC_RHEOLOGY_ELASTIC: launch_fused_stress<SNAC_RHEOLOGY_ELASTIC>(h, F, c); break;
        case SNAC_RHEOLOGY_PLASTIC: launch_fused_stress<SNAC_RHEOLOGY_PLASTIC>(h, F, c); break;
        case SNAC_RHEOLOGY_VISCOPLASTIC:
            if (h->dp)
                launch_fused_stress<SNAC_VP_DP>(h, F, c);
            else
                launch_fused_stress<SNAC_RHEOLOGY_VISCOPLASTIC>(h, F, c);
            break;
        case SNAC_RHEOLOGY_MAXWELL: launch_fused_stress<SNAC_RHEOLOGY_MAXWELL>(h, F, c); break;
    }
    h->launches++;
    return launch_check_named(h, "k_fused_stress");
}

int op_energy_nodes(snac_gpu* h, int count_step = 0) {
    if (!h->temperature) return 0;
    k_heat_nodes<<<node_blocks(h->mesh), 128, 0, h->stream>>>(h->mesh, fields(h), h->cfg, count_step);
    h->launches++;
    if (count_step) h->time_step++;
    return launch_check_named(h, "k_heat_nodes");
}

int op_calc_stresses(snac_gpu* h) {
    Fields F = fields(h);
    switch (h->constitutive) {
        case SNAC_RHEOLOGY_ELASTIC: launch_stress<SNAC_RHEOLOGY_ELASTIC>(h, F, h->cfg); break;
        case SNAC_RHEOLOGY_PLASTIC: launch_stress<SNAC_RHEOLOGY_PLASTIC>(h, F, h->cfg); break;
        case SNAC_RHEOLOGY_VISCOPLASTIC:
            if (h->dp)
                launch_stress<SNAC_VP_DP>(h, F, h->cfg);
            else
                launch_stress<SNAC_RHEOLOGY_VISCOPLASTIC>(h, F, h->cfg);
            break;
        case SNAC_RHEOLOGY_MAXWELL: launch_stress<SNAC_RHEOLOGY_MAXWELL>(h, F, h->cfg); break;
    }
    h->launches++;
    return launch_check_named(h, "k_calc_stresses");
}

int op_loop_nodes(snac_gpu* h) {
    Fields F = fields(h);
    const unsigned nb = node_blocks(h->mesh);
    const bool vo = h->cfg.vonly != 0;
    switch (h->cfg.dt_type) {
        case SNAC_DT_CONSTANT:
            k_loop_nodes<SNAC_DT_CONSTANT, false><<<nb, 128, 0, h->stream>>>(h->mesh, F, h->cfg);
            break;
        case SNAC_DT_DYNAMIC:
            if (vo) k_loop_nodes<SNAC_DT_DYNAMIC, true><<<nb, 128, 0, h->stream>>>(h->mesh, F, h->cfg);
            else k_loop_nodes<SNAC_DT_DYNAMIC, false><<<nb, 128, 0, h->stream>>>(h->mesh, F, h->cfg);
            break;
        default:
            if (vo) k_loop_nodes<SNAC_DT_WAVE, true><<<nb, 128, 0, h->stream>>>(h->mesh, F, h->cfg);
            else k_loop_nodes<SNAC_DT_WAVE, false><<<nb, 128, 0, h->stream>>>(h->mesh, F, h->cfg);
            break;
    }
    h->launches++;
    h->parity ^= 1;  // the new coordinates are current from here on
    int rc = launch_check_named(h, "k_loop_nodes");
    if (rc || !topo_on(h->cfg)) return rc;
    k_topo<<<1, 1024, 0, h->stream>>>(h->mesh, h->pos[h->parity ^ 1], h->pos[h->parity], h->cfg, h->sc, h->topo_scratch);
    h->launches++;
    return launch_check_named(h, "k_topo");
}

int op_update_elements(snac_gpu* h, bool step_zero, int pending = 0) {
    Fields F = fields(h);
    Config c = h->cfg;
    c.time_step_zero = step_zero ? 1 : 0;
    switch (h->constitutive) {
        case SNAC_RHEOLOGY_MAXWELL: launch_update<SNAC_RHEOLOGY_MAXWELL>(h, F, c, pending); break;
        default: launch_update<SNAC_RHEOLOGY_ELASTIC>(h, F, c, pending); break;
    }
    h->launches++;
    return launch_check_named(h, "k_update_elements");
}

// the end of the previous step fused with the start of this one (runs
// without temperature: no energy hook sits between the two)
int op_fused(snac_gpu* h) {
    Fields F = fields(h);
    Config c = h->cfg;
    c.time_step_zero = 0;
    switch (h->constitutive) {
        case SNAC_RHEOLOGY_ELASTIC: launch_fused<SNAC_RHEOLOGY_ELASTIC>(h, F, c); break;
        case SNAC_RHEOLOGY_PLASTIC: launch_fused<SNAC_RHEOLOGY_PLASTIC>(h, F, c); break;
        case SNAC_RHEOLOGY_VISCOPLASTIC:
            if (h->dp)
                launch_fused<SNAC_VP_DP>(h, F, c);
            else
                launch_fused<SNAC_RHEOLOGY_VISCOPLASTIC>(h, F, c);
            break;
        case SNAC_RHEOLOGY_MAXWELL: launch_fused<SNAC_RHEOLOGY_MAXWELL>(h, F, c); break;
    }
    h->launches++;
    h->time_step++;
    return launch_check_named(h, "k_fused_step");
}

int op_min_length_scale_sync(snac_gpu* h) {
    if (h->temperature) {  // with the heat flux of the next step
        if (h->mat)
            k_heat_flux_min_length_scale<false><<<elem_blocks(h->mesh), ELEM_WARPS * 32, 0, h->stream>>>(
                h->mesh, fields(h), h->cfg);
        else
            k_heat_flux_min_length_scale<true><<<elem_blocks(h->mesh), ELEM_WARPS * 32, 0, h->stream>>>(
                h->mesh, fields(h), h->cfg);
        h->launches++;
        int rc = launch_check_named(h, "k_heat_flux_min_length_scale");
        if (rc) return rc;
        k_slots_sync<<<1, 32, 0, h->stream>>>(h->cfg, h->sc, h->wave_speed);
        h->launches++;
        return launch_check_named(h, "k_slots_sync");
    }
    k_min_length_scale_sync<<<(unsigned)((h->mesh.ne + MINLS_THREADS - 1) / MINLS_THREADS), MINLS_THREADS, 0,
                              h->stream>>>(h->mesh, fields(h), h->cfg, h->wave_speed);
    h->launches++;
    return launch_check_named(h, "k_min_length_scale_sync");
}

int op_sync(snac_gpu* h) {
    k_sync<<<1, 32, 0, h->stream>>>(h->cfg, h->sc, h->wave_speed);
    h->launches++;
    return launch_check_named(h, "k_sync");
}

// Sync when the node loop did not just reduce max |v| (step zero, hook by hook)
int op_sync_full(snac_gpu* h) {
    k_vmax<<<(unsigned)((h->mesh.nn + 255) / 256), 256, 0, h->stream>>>(h->mesh, fields(h));
    h->launches++;
    int rc = launch_check_named(h, "k_vmax");
    return rc ? rc : op_sync(h);
}

int op_begin(snac_gpu* h) {
    k_begin_step<<<1, 32, 0, h->stream>>>(h->sc);
    h->launches++;
    h->time_step++;
    return launch_check_named(h, "k_begin_step");
}

// One step as a chain of launches.  Element update of step n and the first
// element kernel of step n+1 share one launch when the previous step's
// update is pending (fused), otherwise the step starts from scratch.
// Temperature runs form the next step's heat flux in the step's last kernel;
// a step whose heat flux is not ready (the first graph step, or one after a
// state change) forms its own first.
int record_step(snac_gpu* h, bool fused) {
    int rc;
    const bool ready = h->temperature && h->hflux_ready;
    if (fused && h->temperature) {
        // heat flux (opens the step; or the temperature update opens it when
        // the flux is ready), temperature update, then the pending element
        // update fused with the stress update
        if (ready) {
            if ((rc = op_energy_nodes(h, 1))) return rc;
        } else {
            if ((rc = op_energy_elements(h, 1))) return rc;
            if ((rc = op_energy_nodes(h))) return rc;
        }
        if ((rc = op_fused_stress(h))) return rc;
    } else if (fused) {
        if ((rc = op_fused(h))) return rc;  // element update + stress update
    } else {
        if ((rc = op_begin(h))) return rc;
        if (!ready && (rc = op_energy_elements(h))) return rc;
        if ((rc = op_energy_nodes(h))) return rc;
        if ((rc = op_calc_stresses(h))) return rc;
    }
    if ((rc = op_loop_nodes(h))) return rc;
    return op_min_length_scale_sync(h);  // temperature runs: with the next step's heat flux
}

// apply a deferred element update so that the state matches the reference's
// end of step (before any transfer or hook-by-hook call)
int flush_pending(snac_gpu* h) {
    if (!h->pending) return 0;
    int rc = op_update_elements(h, false, 1);
    h->pending = false;
    return rc;
}

int read_status(snac_gpu* h) {
    DevScalars s;
    CK(cudaMemcpyAsync(&s, h->sc, sizeof s, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (s.status) {
        const char* what = s.status == SNAC_GPU_ENAN       ? "non-finite value in the state"
                           : s.status == SNAC_GPU_EVOLUME  ? "zero tetrahedron volume"
                           : s.status == SNAC_GPU_EPHYSICS ? "physical check failed (friction angle < 0 or dt_thermal/dt_mech <= 1)"
                           : s.status == SNAC_GPU_EINVAL   ? "softening table must start at plastic strain 0"
                                                           : "device error";
        return set_err(h, s.status, s.err_index, "%s at element/node %lld (time step %lld)", what, s.err_index, s.time_step);
    }
    return 0;
}

// _Snac_Context's isTimeToDump / isTimeToCheckpoint (Context.c:1505-1531)
bool time_to_dump(const OutputState* o, long long ts) {
    return ts == 1 || (ts > 1 && o->dump_every && ts % o->dump_every == 0);
}
bool time_to_checkpoint(const OutputState* o, long long ts) {
    if (ts == (long long)o->max_steps) return true;
    if (ts == 0 || o->checkpoint_every == 0) return false;
    return ts % o->checkpoint_every == 0;
}

// Before step ts runs: ask its stress update to store the element scalars
// when a dump follows it.  A plain stream operation outside any graph.
int request_scalars(snac_gpu* h, long long ts) {
    if (!h->out) return 0;
    const int want = time_to_dump(h->out, ts) ? 1 : 0;
    if (want == h->out->want) return 0;
    CK(cudaMemsetAsync(&h->sc->want_scalars, want, sizeof(int), h->stream));  // any nonzero byte pattern is true
    h->out->want = want;
    return 0;
}

// one step from the handle's CUDA graph for its (pending, parity) state,
// captured on first use; no status read
int launch_step(snac_gpu* h) {
    if (int rc = request_scalars(h, h->time_step + 1)) return rc;
    int p = h->parity, f = h->pending ? 1 : 0, r = (h->temperature && h->hflux_ready) ? 1 : 0;
    if (!h->graph[r][f][p]) {
        cudaGraph_t g;
        long long l0 = h->launches, ts0 = h->time_step;
        CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
        int rc = record_step(h, f == 1);
        cudaError_t e = cudaStreamEndCapture(h->stream, &g);
        if (rc) return rc;
        if (e != cudaSuccess) return set_err(h, SNAC_GPU_ECUDA, -1, "graph capture: %s", cudaGetErrorString(e));
        CK(cudaGraphInstantiate(&h->graph[r][f][p], g, 0));
        cudaGraphDestroy(g);
        h->steps_kernels[r][f] = (int)(h->launches - l0);
        h->launches = l0;  // counted again below, when the graph actually runs
        h->time_step = ts0;
        h->parity = p;
    }
    CK(cudaGraphLaunch(h->graph[r][f][p], h->stream));
    h->launches += h->steps_kernels[r][f];
    h->time_step++;
    h->parity ^= 1;
    h->pending = true;
    h->hflux_ready = h->temperature;
    return 0;
}

// node-field transfers through a device staging buffer of 3 doubles per
// node (allocated on first use), repacked by a kernel on the handle's stream
int ensure_stage(snac_gpu* h) {
    if (h->stage) return 0;
    return dalloc(h, &h->stage, (size_t)h->mesh.nn * 3);
}

int node_in(snac_gpu* h, double4* dst, const double* src, int what) {
    int rc = ensure_stage(h);
    if (rc) return rc;
    const long long nn = h->mesh.nn;
    CK(cudaMemcpyAsync(h->stage, src, nn * (what == 0 ? 3 : 1) * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    k_unpack_nodes<<<(unsigned)((nn + 255) / 256), 256, 0, h->stream>>>(dst, h->stage, nn, what);
    h->launches++;
    return launch_check_named(h, "k_unpack_nodes");
}

int node_out(snac_gpu* h, const double4* src, double* dst, int what) {
    int rc = ensure_stage(h);
    if (rc) return rc;
    const long long nn = h->mesh.nn;
    k_pack_nodes<<<(unsigned)((nn + 255) / 256), 256, 0, h->stream>>>(src, h->stage, nn, what);
    h->launches++;
    if ((rc = launch_check_named(h, "k_pack_nodes"))) return rc;
    CK(cudaMemcpyAsync(dst, h->stage, nn * (what == 0 ? 3 : 1) * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    // the next transfer reuses the staging buffer only after this copy (same stream)
    return 0;
}

// ---- slab launches of snac_gpu_step_host -----------------------------------------
// Element slabs are block ranges [b0, b1) of the whole-mesh element launch,
// node slabs block ranges of the node launch; an empty range launches nothing.
int op_calc_stresses_slab(snac_gpu* h, const Fields& F, int b0, int b1) {
    if (b1 <= b0) return 0;
    const unsigned nb = (unsigned)(b1 - b0);
    const Config& c = h->cfg;
    cudaStream_t st = h->stream;
#define SLAB_STRESS(P)                                                                              \
    do {                                                                                             \
        if (h->mat) k_calc_stresses_slab<P, false><<<nb, ELEM_WARPS * 32, 0, st>>>(h->mesh, F, c, b0); \
        else k_calc_stresses_slab<P, true><<<nb, ELEM_WARPS * 32, 0, st>>>(h->mesh, F, c, b0);         \
    } while (0)
    switch (h->constitutive) {
        case SNAC_RHEOLOGY_ELASTIC: SLAB_STRESS(SNAC_RHEOLOGY_ELASTIC); break;
        case SNAC_RHEOLOGY_PLASTIC: SLAB_STRESS(SNAC_RHEOLOGY_PLASTIC); break;
        case SNAC_RHEOLOGY_VISCOPLASTIC:
            if (h->dp) SLAB_STRESS(SNAC_VP_DP);
            else SLAB_STRESS(SNAC_RHEOLOGY_VISCOPLASTIC);
            break;
        case SNAC_RHEOLOGY_MAXWELL: SLAB_STRESS(SNAC_RHEOLOGY_MAXWELL); break;
    }
#undef SLAB_STRESS
    h->launches++;
    return launch_check_named(h, "k_calc_stresses_slab");
}

int op_loop_nodes_slab(snac_gpu* h, const Fields& F, int b0, int b1) {
    if (b1 <= b0) return 0;
    const unsigned nb = (unsigned)(b1 - b0);
    const bool vo = h->cfg.vonly != 0;
    cudaStream_t st = h->stream;
    switch (h->cfg.dt_type) {
        case SNAC_DT_CONSTANT:
            k_loop_nodes_slab<SNAC_DT_CONSTANT, false><<<nb, 128, 0, st>>>(h->mesh, F, h->cfg, b0);
            break;
        case SNAC_DT_DYNAMIC:
            if (vo) k_loop_nodes_slab<SNAC_DT_DYNAMIC, true><<<nb, 128, 0, st>>>(h->mesh, F, h->cfg, b0);
            else k_loop_nodes_slab<SNAC_DT_DYNAMIC, false><<<nb, 128, 0, st>>>(h->mesh, F, h->cfg, b0);
            break;
        default:
            if (vo) k_loop_nodes_slab<SNAC_DT_WAVE, true><<<nb, 128, 0, st>>>(h->mesh, F, h->cfg, b0);
            else k_loop_nodes_slab<SNAC_DT_WAVE, false><<<nb, 128, 0, st>>>(h->mesh, F, h->cfg, b0);
            break;
    }
    h->launches++;
    return launch_check_named(h, "k_loop_nodes_slab");
}

int op_update_elements_slab(snac_gpu* h, const Fields& F, int b0, int b1) {
    if (b1 <= b0) return 0;
    const unsigned nb = (unsigned)(b1 - b0);
    Config c = h->cfg;
    c.time_step_zero = 0;
    if (h->constitutive == SNAC_RHEOLOGY_MAXWELL)
        k_update_elements_slab<SNAC_RHEOLOGY_MAXWELL><<<nb, ELEM_WARPS * 32, 0, h->stream>>>(h->mesh, F, c, b0);
    else
        k_update_elements_slab<SNAC_RHEOLOGY_ELASTIC><<<nb, ELEM_WARPS * 32, 0, h->stream>>>(h->mesh, F, c, b0);
    h->launches++;
    return launch_check_named(h, "k_update_elements_slab");
}

int op_heat_flux_slab(snac_gpu* h, const Fields& F, int b0, int b1) {
    if (b1 <= b0) return 0;
    const unsigned nb = (unsigned)(b1 - b0);
    if (h->mat)
        k_heat_flux_slab<false><<<nb, ELEM_WARPS * 32, 0, h->stream>>>(h->mesh, F, h->cfg, b0);
    else
        k_heat_flux_slab<true><<<nb, ELEM_WARPS * 32, 0, h->stream>>>(h->mesh, F, h->cfg, b0);
    h->launches++;
    return launch_check_named(h, "k_heat_flux_slab");
}

int op_heat_nodes_slab(snac_gpu* h, const Fields& F, int b0, int b1) {
    if (b1 <= b0) return 0;
    k_heat_nodes_slab<<<(unsigned)(b1 - b0), 128, 0, h->stream>>>(h->mesh, F, h->cfg, b0);
    h->launches++;
    return launch_check_named(h, "k_heat_nodes_slab");
}

int ensure_host_step(snac_gpu* h) {
    if (h->hs && h->hs->ready) return 0;
    if (h->hs) return set_err(h, SNAC_GPU_ESTATE, -1, "snac_gpu_step_host: an earlier set-up of its streams failed");
    HostStep* q = new HostStep();
    h->hs = q;  // released by snac_gpu_destroy, also when set-up fails half way
    CK(cudaStreamCreateWithFlags(&q->in, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&q->out, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&q->start, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&q->done, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&q->nodes_in, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&q->nodes_rest, cudaEventDisableTiming));
    for (int c = 0; c < STEP_HOST_MAX_CHUNKS; c++) {
        CK(cudaEventCreateWithFlags(&q->ev_in[c], cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&q->ev_elems[c], cudaEventDisableTiming));
    }
    int rc;
    if ((rc = dalloc(h, &q->stage_in, (size_t)h->mesh.nn * 7))) return rc;
    if ((rc = dalloc(h, &q->stage_out, (size_t)h->mesh.nn * 7))) return rc;
    q->ready = true;
    return 0;
}

// hydroStaticIC/VariableConditions.c:43-152 on one rank: lithostatic
// pressure integrated down each element column; densities are the phase
// densities (tet densities are still zero at this point of the reference's IC).
// returns pisos, the bottom pressure of column (0, 0) (:133-140)
double hydrostatic_ic(const snac_gpu_desc* d, const std::vector<double>& coord, std::vector<double>& stress) {
    double pisos = 0.0;
    int nx = d->nx, ny = d->ny, nz = d->nz, nnx = nx + 1, nny = ny + 1;
    auto y_of = [&](long e, int corner) {
        static const int off[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
        int i = (int)(e % nx), j = (int)((e / nx) % ny), k = (int)(e / ((long)nx * ny));
        long n = (i + off[corner][0]) + (long)(j + off[corner][1]) * nnx + (long)(k + off[corner][2]) * nnx * nny;
        return coord[n * 3 + 1];
    };
    for (int elK = 0; elK < nz; elK++)
        for (int elI = 0; elI < nx; elI++) {
            double rogh = 0.0f;
            for (int elJ = ny - 1; elJ > -1; elJ--) {
                long e = elI + (long)elJ * nx + (long)elK * nx * ny;
                int ph = d->element_material ? d->element_material[e] : 0;
                const snac_material& m = d->materials[ph];
                double densT = 0.0f;
                for (int t = 0; t < NT; t++) densT += (m.density * (1.0 - m.alpha * (0.0 - m.reftemp))) / NT;
                double dhE[4];
                dhE[0] = y_of(e, 6) - y_of(e, 0);
                dhE[1] = y_of(e, 2) - y_of(e, 4);
                dhE[2] = y_of(e, 3) - y_of(e, 5);
                dhE[3] = y_of(e, 7) - y_of(e, 1);
                double dh = 0.25f * (dhE[0] + dhE[1] + dhE[2] + dhE[3]);
                double dPT = densT * d->gravity * dh;
                double dP = dPT * (1.0 - m.beta * rogh) / (1.0f + m.beta / 2.0f * dPT);
                double P = rogh + 0.5f * dP;
                P = -1.0f * (P + 0.0);
                for (int t = 0; t < NT; t++)
                    for (int c = 0; c < 3; c++) stress[((size_t)e * NT + t) * 6 + c] = P;
                rogh += dP;
                if (elJ == 0 && elI == 0 && elK == 0) pisos = rogh + 0.0;
            }
        }
    return pisos;
}

}  // namespace

extern "C" {

int snac_gpu_selftest_division(long long n, unsigned long long seed, long long* mismatches) {
    if (!mismatches || n < 0) return SNAC_GPU_EINVAL;
    unsigned long long* d = nullptr;
    if (cudaMalloc(&d, sizeof *d) != cudaSuccess) return SNAC_GPU_ENOMEM;
    cudaMemset(d, 0, sizeof *d);
    k_selftest_division<<<148 * 8, 256>>>(n, seed, d);
    unsigned long long h = 0;
    cudaError_t e = cudaMemcpy(&h, d, sizeof h, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return SNAC_GPU_ECUDA;
    *mismatches = (long long)h;
    return 0;
}

// FP64 throughput of this GPU: eight independent FMA chains per thread, the
// grid a multiple of the SM count.  The result never equals the sentinel for
// these inputs (every chain converges to c / (1 - b) = 1e3), so the chains
// stay live and the store never happens.
__global__ void k_fp64_rate(int iters, double b, double c, double* sink) {
    double a[8];
#pragma unroll
    for (int k = 0; k < 8; k++) a[k] = 1.0 + 1.0e-3 * (double)(threadIdx.x + k);
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 8; k++) a[k] = fma(a[k], b, c);
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 8; k++) s += a[k];
    if (s == -1.0) sink[0] = s;
}

int snac_gpu_fp64_rate(double* fma_per_second) {
    if (!fma_per_second) return SNAC_GPU_EINVAL;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return SNAC_GPU_ENODEV;
    double* sink = nullptr;
    if (cudaMalloc(&sink, sizeof(double)) != cudaSuccess) return SNAC_GPU_ENOMEM;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    const int iters = 4096, threads = 256, blocks = sms * 8;
    double best = 0.0;
    cudaError_t e = cudaSuccess;
    for (int rep = 0; rep < 4 && e == cudaSuccess; rep++) {  // the first launch warms up
        cudaEventRecord(a);
        k_fp64_rate<<<blocks, threads>>>(iters, 0.999, 1.0, sink);
        cudaEventRecord(b);
        e = cudaEventSynchronize(b);
        float ms = 0.0f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
        if (rep > 0 && e == cudaSuccess && ms > 0.0f) {
            const double rate = (double)blocks * threads * 8.0 * iters / (ms * 1.0e-3);
            if (rate > best) best = rate;
        }
    }
    if (e == cudaSuccess) e = cudaGetLastError();
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(sink);
    if (e != cudaSuccess) return SNAC_GPU_ECUDA;
    *fma_per_second = best;
    return 0;
}

int snac_gpu_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
    return n;
}

// Builds a model; with shared != null the model uses that stream (batches)
static int create_model(const snac_gpu_desc* d_in, snac_gpu** out, cudaStream_t shared) {
    if (!out) return SNAC_GPU_EINVAL;
    *out = nullptr;
    if (!d_in || (d_in->abi_version != 1 && d_in->abi_version != SNAC_GPU_ABI_VERSION)) return SNAC_GPU_EINVAL;
    // a version-1 descriptor ends at topo_grad_criterion: the version-2 fields read as zero
    snac_gpu_desc dv;
    memset(&dv, 0, sizeof dv);
    memcpy(&dv, d_in, d_in->abi_version == 1 ? offsetof(snac_gpu_desc, pisos) : sizeof dv);
    const snac_gpu_desc* d = &dv;
    if (d->nx < 1 || d->ny < 1 || d->nz < 1 || d->n_materials < 1 || !d->materials) return SNAC_GPU_EINVAL;
    if (d->n_materials > MAX_PHASES) return SNAC_GPU_EINVAL;
    if (d->constitutive != SNAC_RHEOLOGY_ELASTIC && d->constitutive != SNAC_RHEOLOGY_PLASTIC &&
        d->constitutive != SNAC_RHEOLOGY_VISCOPLASTIC && d->constitutive != SNAC_RHEOLOGY_MAXWELL)
        return SNAC_GPU_EINVAL;
    if ((d->constitutive == SNAC_RHEOLOGY_VISCOPLASTIC || d->constitutive == SNAC_RHEOLOGY_MAXWELL) && !d->temperature)
        return SNAC_GPU_EINVAL;  // both hooks read the temperature plugin's node extension
    if (d->dt_type < SNAC_DT_CONSTANT || d->dt_type > SNAC_DT_WAVE) return SNAC_GPU_EINVAL;
    if ((d->topo_kappa > 0 || !(d->topo_grad_criterion > 0)) && (d->nx < 2 || d->nz < 2))
        return SNAC_GPU_ENOTSUP;  // diffTopo_alongX / alongZ (one element wide) are not built
    bool per_elem = d->element_cohesion_scale || d->element_friction_scale || d->element_visc_scale;
    if (per_elem && d->constitutive == SNAC_RHEOLOGY_MAXWELL) return SNAC_GPU_ENOTSUP;
    for (int p = 0; p < d->n_materials; p++) {
        if (d->materials[p].nsegments < 0 || d->materials[p].nsegments > SNAC_MAX_SEGMENTS) return SNAC_GPU_EINVAL;
        if (d->dp_max_iterations && d->dp_max_iterations[p] < 0) return SNAC_GPU_EINVAL;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return SNAC_GPU_ENODEV;
    for (int b = 0; b < d->n_velocity_bcs; b++)
        if (d->velocity_bcs[b].wall < 0 || d->velocity_bcs[b].wall > SNAC_WALL_ALL) return SNAC_GPU_EINVAL;
    if (d->n_velocity_bcs > 254 || d->n_temperature_bcs > 254) return SNAC_GPU_EINVAL;

    snac_gpu* h = new (std::nothrow) snac_gpu();
    if (!h) return SNAC_GPU_ENOMEM;
    *out = h;
    Mesh& m = h->mesh;
    m.nx = d->nx;
    m.ny = d->ny;
    m.nz = d->nz;
    m.nnx = d->nx + 1;
    m.nny = d->ny + 1;
    m.nnz = d->nz + 1;
    m.ne = (long long)d->nx * d->ny * d->nz;
    m.nn = (long long)m.nnx * m.nny * m.nnz;
    m.ner = (m.ne + 3) & ~3LL;
    h->constitutive = d->constitutive;
    h->temperature = d->temperature;
    h->abi = d_in->abi_version;
    if (d->constitutive == SNAC_RHEOLOGY_VISCOPLASTIC)  // only the visco-plastic hook has the Drucker-Prager branch
        for (int p = 0; p < d->n_materials; p++)
            if (!d->materials[p].yield_mohr_coulomb) h->dp = 1;
    h->n_phases = d->n_materials;
    for (int p = 0; p < d->n_materials; p++)
        if (d->materials[p].alpha != 0.0 || d->materials[p].beta != 0.0) h->has_density = 1;
    Config& c = h->cfg;
    c.dt_type = d->dt_type;
    c.constitutive = d->constitutive;
    c.temperature = d->temperature;
    c.thermal_stress = d->compute_thermal_stress && d->temperature;
    c.has_density = h->has_density;
    c.gravity = d->gravity;
    c.demf = d->demf;
    c.strain_inert = d->strain_inert;
    c.winkler = d->winkler ? 1 : 0;
    c.traction = d->traction_bc ? 1 : 0;
    c.topo_kappa = d->topo_kappa;
    c.topo_crit = d->topo_grad_criterion;
    {
        int dev = 0, sms = 0;
        if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess)
            c.prefetch_ahead = sms * SNAC_ELEM_MINB;
    }
    c.pisos = d->pisos;  // replaced below when the hydrostatic IC runs here
    c.rzbo = d->rzbo;
    if (shared) {
        h->stream = shared;
        h->own_stream = false;
    } else {
        CK(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    }

    const long long ne = m.ne, nn = m.nn, nq = ne * NT;
    int rc = 0;
    if ((rc = dalloc(h, &h->pos[0], nn)) || (rc = dalloc(h, &h->pos[1], nn)) || (rc = dalloc(h, &h->vel, nn)) ||
        (rc = dalloc(h, &h->force, nn)) || (rc = dalloc(h, &h->stress, nq * 6)) || (rc = dalloc(h, &h->bc, nn)) ||
        (rc = dalloc(h, &h->sc, 1)) || (rc = dalloc(h, &h->mats, MAX_PHASES)) ||
        (rc = dalloc(h, &h->fterm, m.ner * NT * 12)) || (rc = dalloc(h, &h->fgrav, m.ner * NT)) ||
        (rc = dalloc(h, &h->fmass, m.ner * NT * (d->dt_type == SNAC_DT_CONSTANT ? 4 : 1))))
        return rc;
    if (d->constitutive == SNAC_RHEOLOGY_PLASTIC || d->constitutive == SNAC_RHEOLOGY_VISCOPLASTIC)
        if ((rc = dalloc(h, &h->eps_p, nq))) return rc;
    if (d->constitutive == SNAC_RHEOLOGY_VISCOPLASTIC || d->constitutive == SNAC_RHEOLOGY_MAXWELL)
        if ((rc = dalloc(h, &h->visc, nq))) return rc;
    if (h->dp && (rc = dalloc(h, &h->pst, nq * 6))) return rc;
    if (d->constitutive == SNAC_RHEOLOGY_MAXWELL)
        if ((rc = dalloc(h, &h->vol, nq * 2))) return rc;
    if (h->has_density)
        if ((rc = dalloc(h, &h->density, nq))) return rc;
    if (d->winkler)
        if ((rc = dalloc(h, &h->residual_fr, nn))) return rc;
    if (topo_on(c))
        if ((rc = dalloc(h, &h->topo_scratch, (size_t)m.nnx * m.nnz))) return rc;
    if (d->temperature) {
        if ((rc = dalloc(h, &h->hflux, m.ner * NT * HF_STRIDE))) return rc;
        if (h->has_density && (rc = dalloc(h, &h->tpre, nn))) return rc;
    }

    // ---- conditions resolved per node (ABI 2): one table entry per distinct value ----
    // entry b of the velocity table holds, for each component q, the b-th
    // distinct value of that component; a node's index per component points there
    std::vector<std::vector<double>> pn_vval(3);
    std::vector<double> pn_tval;
    auto slot_of = [](std::vector<double>& vals, double v) -> int {
        for (size_t b = 0; b < vals.size(); b++)
            if (memcmp(&vals[b], &v, sizeof v) == 0) return (int)b;
        vals.push_back(v);
        return (int)vals.size() - 1;
    };
    std::vector<uchar4> pn_idx;
    if (d->node_velocity_bc_mask || d->node_temperature_bc_mask) {
        pn_idx.assign(nn, make_uchar4(255, 255, 255, 255));
        for (long long n = 0; n < nn; n++) {
            unsigned char idx[4] = {255, 255, 255, 255};
            for (int q = 0; q < 3; q++)
                if (d->node_velocity_bc_mask && (d->node_velocity_bc_mask[n] & (1 << q))) {
                    int b = slot_of(pn_vval[q], d->node_velocity_bc_value[n * 3 + q]);
                    if (b > 253) return set_err(h, SNAC_GPU_ENOTSUP, n, "more than 254 distinct velocity-BC values");
                    idx[q] = (unsigned char)b;
                }
            if (d->temperature && d->node_temperature_bc_mask && d->node_temperature_bc_mask[n]) {
                int b = slot_of(pn_tval, d->node_temperature_bc_value[n]);
                if (b > 253) return set_err(h, SNAC_GPU_ENOTSUP, n, "more than 254 distinct temperature-BC values");
                idx[3] = (unsigned char)b;
            }
            pn_idx[n] = make_uchar4(idx[0], idx[1], idx[2], idx[3]);
        }
    }
    const bool pn_vel = d->node_velocity_bc_mask != nullptr, pn_temp = d->node_temperature_bc_mask != nullptr;

    // ---- initial conditions on the host ----
    std::vector<double> coord(nn * 3), vel(nn * 3, 0.0), temp(nn, 0.0), temp0(nn, 0.0), stress(nq * 6, 0.0);
    std::vector<uchar4> bc(nn, make_uchar4(255, 255, 255, 255));
    for (long long n = 0; n < nn; n++) {
        int i = (int)(n % m.nnx), j = (int)((n / m.nnx) % m.nny), k = (int)(n / ((long long)m.nnx * m.nny));
        int ijk[3] = {i, j, k}, size[3] = {m.nnx, m.nny, m.nnz};
        for (int q = 0; q < 3; q++) {
            // BlockGeometry.c:326-349
            coord[n * 3 + q] = d->node_coords ? d->node_coords[n * 3 + q]
                               : size[q] > 1  ? d->min[q] + (d->max[q] - d->min[q]) * ((double)ijk[q] / (double)(size[q] - 1))
                                              : d->min[q];
            if (d->init_velocity) vel[n * 3 + q] = d->init_velocity[n * 3 + q];
        }
        if (d->temperature) {
            if (d->temperature_sweep_ic)  // temperature/VariableConditions.c:52-73
                temp[n] = d->bottom_temp + (d->top_temp - d->bottom_temp) / (m.nny - 1) * j;
            else if (d->init_temperature)
                temp[n] = d->init_temperature[n];
        }
        unsigned char idx[4] = {255, 255, 255, 255};
        if (!pn_vel)
            for (int b = 0; b < d->n_velocity_bcs; b++) {  // last VC wins, CompositeVC.c:599-611
                const snac_wall_bc& w = d->velocity_bcs[b];
                if (!wall_has(w.wall, i, j, k, m.nnx, m.nny, m.nnz)) continue;
                for (int q = 0; q < 3; q++)
                    if (w.mask & (1 << q)) idx[q] = (unsigned char)b;
            }
        else
            for (int q = 0; q < 3; q++) idx[q] = (&pn_idx[n].x)[q];
        if (!pn_temp)
            for (int b = 0; b < d->n_temperature_bcs; b++) {
                const snac_wall_bc& w = d->temperature_bcs[b];
                if ((w.mask & 1) && wall_has(w.wall, i, j, k, m.nnx, m.nny, m.nnz)) idx[3] = (unsigned char)b;
            }
        else
            idx[3] = pn_idx[n].w;
        bc[n] = make_uchar4(idx[0], idx[1], idx[2], idx[3]);
        // temperature0 = temperature before the BCs are applied
        // (_SnacTemperature_InitialConditions, temperature/VariableConditions.c:240-256)
        temp0[n] = temp[n];
        // VariableCondition_Apply(velocityBCs), Context.c:773
        for (int q = 0; q < 3; q++)
            if (idx[q] != 255) vel[n * 3 + q] = pn_vel ? pn_vval[q][idx[q]] : d->velocity_bcs[idx[q]].value[q];
        if (d->temperature && idx[3] != 255) temp[n] = pn_temp ? pn_tval[idx[3]] : d->temperature_bcs[idx[3]].value[0];
    }
    if (d->init_stress) std::copy(d->init_stress, d->init_stress + nq * 6, stress.begin());
    if (d->hydrostatic_ic) {
        h->cfg.pisos = hydrostatic_ic(d, coord, stress);
        h->cfg.rzbo = d->min[1];  // element->rzbo = geometry->min[1]
    }

    std::vector<double4> pos4(nn), vel4(nn);
    for (long long n = 0; n < nn; n++) {
        pos4[n] = make_double4(coord[n * 3], coord[n * 3 + 1], coord[n * 3 + 2], temp[n]);
        vel4[n] = make_double4(vel[n * 3], vel[n * 3 + 1], vel[n * 3 + 2], temp0[n]);
    }
    const int nvb = pn_vel ? (int)std::max(pn_vval[0].size(), std::max(pn_vval[1].size(), pn_vval[2].size()))
                           : d->n_velocity_bcs;
    const int ntb = pn_temp ? (int)pn_tval.size() : d->n_temperature_bcs;
    std::vector<double> vbc(std::max(1, nvb) * 3, 0.0), tbc(std::max(1, ntb), 0.0);
    for (int b = 0; b < nvb; b++)
        for (int q = 0; q < 3; q++)
            vbc[b * 3 + q] = pn_vel ? (b < (int)pn_vval[q].size() ? pn_vval[q][b] : 0.0) : d->velocity_bcs[b].value[q];
    for (int b = 0; b < ntb; b++) tbc[b] = pn_temp ? pn_tval[b] : d->temperature_bcs[b].value[0];
    if ((rc = dalloc(h, &h->vbc_val, vbc.size())) || (rc = dalloc(h, &h->tbc_val, tbc.size()))) return rc;

    std::vector<DevMaterial> dm(MAX_PHASES);
    for (int p = 0; p < d->n_materials; p++)  // Drucker-Prager controls: Context.c:851-854 defaults 1 and 1e-3
        dm[p] = to_dev(d->materials[p], d->element_friction_scale != nullptr,
                       d->dp_max_iterations ? d->dp_max_iterations[p] : 1, d->dp_tolerance ? d->dp_tolerance[p] : 1.e-3);
    // the volume alone stands for the gravity and inertial-mass terms (Config::vonly)
    h->cfg.vonly = SNAC_VOLUME_ONLY && !d->element_material && !h->has_density && d->dt_type != SNAC_DT_CONSTANT;
    if (d->element_material) {
        std::vector<unsigned char> mt(ne);
        for (long long e = 0; e < ne; e++) {
            int p = d->element_material[e];
            if (p < 0 || p >= d->n_materials) return set_err(h, SNAC_GPU_EMATERIAL, e, "element %lld: phase %d out of range", e, p);
            mt[e] = (unsigned char)p;
        }
        if ((rc = dalloc(h, &h->mat, ne))) return rc;
        CK(cudaMemcpyAsync(h->mat, mt.data(), ne, cudaMemcpyHostToDevice, h->stream));
    }
    auto up_scale = [&](const double* src, double** dst) -> int {
        if (!src) return 0;
        int r = dalloc(h, dst, ne);
        if (r) return r;
        CK(cudaMemcpyAsync(*dst, src, ne * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        return 0;
    };
    if ((rc = up_scale(d->element_cohesion_scale, &h->coh_scale)) || (rc = up_scale(d->element_friction_scale, &h->fric_scale)) ||
        (rc = up_scale(d->element_visc_scale, &h->visc_scale)))
        return rc;

    // plugin ICs: visco-plastic viscosity = vis_min and the Maxwell-time dt bounds
    DevScalars sc;
    memset(&sc, 0, sizeof sc);
    sc.dt = d->dt;
    sc.minls_bits = 0x7ff0000000000000ull;
    for (auto& b : sc.minls_slot) b = 0x7ff0000000000000ull;
    if (d->constitutive == SNAC_RHEOLOGY_VISCOPLASTIC) {  // viscoplastic/InitialConditions.c:49-90
        double dtm = 0;
        for (int p = 0; p < d->n_materials; p++) {
            double v = 9.0e-01 * d->materials[p].vis_min / d->materials[p].mu;
            dtm = (p == 0) ? v : std::min(v, dtm);
        }
        if (sc.dt > dtm && d->dt_type != SNAC_DT_CONSTANT) sc.dt = dtm;
        std::vector<double> v0(nq);
        for (long long e = 0; e < ne; e++) {
            int p = d->element_material ? d->element_material[e] : 0;
            for (int t = 0; t < NT; t++) v0[e * NT + t] = d->materials[p].vis_min;
        }
        CK(cudaMemcpyAsync(h->visc, v0.data(), nq * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    }
    if (d->constitutive == SNAC_RHEOLOGY_MAXWELL) {  // maxwell/InitialConditions.c:43-67
        double dtm = 1.0e-01 * d->materials[0].vis_min / d->materials[0].mu;
        if (sc.dt > dtm && d->dt_type != SNAC_DT_CONSTANT) sc.dt = dtm;
    }
    if (d->dt_type == SNAC_DT_WAVE) {  // running max of Vp, UpdateElement.c:64-69
        double w = 0.0;
        for (long long e = 0; e < ne; e++) {
            const snac_material& mm = d->materials[d->element_material ? d->element_material[e] : 0];
            double Vp = sqrt((mm.lambda + 2.0f * mm.mu) / mm.density);
            if (Vp > w) w = Vp;
        }
        h->wave_speed = w;
    }
    CK(cudaMemcpyAsync(h->pos[0], pos4.data(), nn * sizeof(double4), cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->vel, vel4.data(), nn * sizeof(double4), cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->stress, stress.data(), nq * 6 * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->bc, bc.data(), nn * sizeof(uchar4), cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->vbc_val, vbc.data(), vbc.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->tbc_val, tbc.data(), tbc.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->mats, dm.data(), MAX_PHASES * sizeof(DevMaterial), cudaMemcpyHostToDevice, h->stream));
    h->cfg.m0 = dm[0];
    CK(cudaMemcpyAsync(h->sc, &sc, sizeof sc, cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return 0;
}

int snac_gpu_create(const snac_gpu_desc* d, snac_gpu** out) { return create_model(d, out, nullptr); }

int snac_gpu_output_close(snac_gpu* h);

void snac_gpu_destroy(snac_gpu* h) {
    if (!h) return;
    snac_gpu_output_close(h);
    if (h->stream) cudaStreamSynchronize(h->stream);
    for (auto& gr : h->graph)
        for (auto& gf : gr)
            for (auto& g : gf)
                if (g) cudaGraphExecDestroy(g);
    if (HostStep* q = h->hs) {
        for (cudaStream_t st : {q->in, q->out})
            if (st) cudaStreamSynchronize(st);
        for (cudaEvent_t e : {q->start, q->done, q->nodes_in, q->nodes_rest})
            if (e) cudaEventDestroy(e);
        for (int c = 0; c < STEP_HOST_MAX_CHUNKS; c++)
            for (cudaEvent_t e : {q->ev_in[c], q->ev_elems[c]})
                if (e) cudaEventDestroy(e);
        for (cudaStream_t st : {q->in, q->out})
            if (st) cudaStreamDestroy(st);
        if (q->stage_in) cudaFree(q->stage_in);
        if (q->stage_out) cudaFree(q->stage_out);
        delete q;
    }
    void* bufs[] = {h->pos[0], h->pos[1], h->vel, h->force, h->stress, h->eps_p, h->pst, h->visc, h->density, h->vol,
                    h->hflux, h->tpre, h->fterm, h->fgrav, h->fmass, h->bc, h->vbc_val, h->tbc_val, h->mat, h->mats, h->coh_scale, h->fric_scale,
                    h->visc_scale, h->sc, h->stage, h->escal, h->residual_fr, h->topo_scratch};
    for (void* b : bufs)
        if (b) cudaFree(b);
    if (h->stream && h->own_stream) cudaStreamDestroy(h->stream);
    delete h;
}

int snac_gpu_time_step_zero(snac_gpu* h) {
    if (!h) return SNAC_GPU_EINVAL;
    h->hflux_ready = false;  // the state or the step sequence changes
    if (h->zero_done) return set_err(h, SNAC_GPU_ESTATE, -1, "time step zero already done");
    // Context.c:999-1020: tet density = phase density (the element scalar stress is an output only)
    if (h->has_density) {
        std::vector<double> rho(h->mesh.ne * NT);
        std::vector<unsigned char> mt;
        std::vector<DevMaterial> dm(MAX_PHASES);
        CK(cudaMemcpy(dm.data(), h->mats, MAX_PHASES * sizeof(DevMaterial), cudaMemcpyDeviceToHost));
        if (h->mat) {
            mt.resize(h->mesh.ne);
            CK(cudaMemcpy(mt.data(), h->mat, h->mesh.ne, cudaMemcpyDeviceToHost));
        }
        for (long long e = 0; e < h->mesh.ne; e++)
            for (int t = 0; t < NT; t++) rho[e * NT + t] = dm[h->mat ? mt[e] : 0].density;
        CK(cudaMemcpyAsync(h->density, rho.data(), rho.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    }
    int rc;
    if ((rc = op_update_elements(h, true))) return rc;
    if ((rc = op_sync_full(h))) return rc;
    h->zero_done = true;
    return read_status(h);
}

int snac_gpu_step(snac_gpu* h, int nsteps) {
    if (!h || nsteps < 0) return SNAC_GPU_EINVAL;
    if (!h->zero_done) return set_err(h, SNAC_GPU_ESTATE, -1, "snac_gpu_time_step_zero must come first");
    for (int s = 0; s < nsteps; s++) {
        int rc = launch_step(h);
        if (rc) return rc;
    }
    return read_status(h);
}

int snac_gpu_time_steps(snac_gpu* h, int nsteps, void* flush, size_t flush_bytes, double* ms) {
    if (!h || nsteps < 1 || !ms || (flush_bytes && !flush)) return SNAC_GPU_EINVAL;
    if (!h->zero_done) return set_err(h, SNAC_GPU_ESTATE, -1, "snac_gpu_time_step_zero must come first");
    std::vector<cudaEvent_t> ev((size_t)nsteps * 2, nullptr);
    int rc = 0;
    for (auto& e : ev)
        if (cudaEventCreate(&e) != cudaSuccess) rc = set_err(h, SNAC_GPU_ECUDA, -1, "cudaEventCreate failed");
    for (int s = 0; s < nsteps && !rc; s++) {
        if (flush_bytes && cudaMemsetAsync(flush, s & 0xff, flush_bytes, h->stream) != cudaSuccess)
            rc = set_err(h, SNAC_GPU_ECUDA, -1, "cudaMemsetAsync of the flush buffer failed");
        if (!rc) cudaEventRecord(ev[2 * s], h->stream);
        if (!rc) rc = launch_step(h);
        if (!rc) cudaEventRecord(ev[2 * s + 1], h->stream);
    }
    if (cudaStreamSynchronize(h->stream) != cudaSuccess && !rc)
        rc = set_err(h, SNAC_GPU_ECUDA, -1, "%s", cudaGetErrorString(cudaGetLastError()));
    for (int s = 0; s < nsteps && !rc; s++) {
        float t = 0.f;
        cudaEventElapsedTime(&t, ev[2 * s], ev[2 * s + 1]);
        ms[s] = t;
    }
    for (auto& e : ev)
        if (e) cudaEventDestroy(e);
    return rc ? rc : read_status(h);
}

int snac_gpu_begin_step(snac_gpu* h) {
    if (!h) return SNAC_GPU_EINVAL;
    h->hflux_ready = false;  // the state or the step sequence changes
    if (int rc = request_scalars(h, h->time_step + 1)) return rc;
    if (!h->zero_done) return set_err(h, SNAC_GPU_ESTATE, -1, "snac_gpu_time_step_zero must come first");
    int rc = flush_pending(h);
    return rc ? rc : op_begin(h);
}
int snac_gpu_loop_elements_energy(snac_gpu* h) {
    if (!h) return SNAC_GPU_EINVAL;
    h->hflux_ready = false;  // the state or the step sequence changes
    int rc = flush_pending(h);
    return rc ? rc : op_energy_elements(h);
}
int snac_gpu_loop_nodes_energy(snac_gpu* h) {
    if (!h) return SNAC_GPU_EINVAL;
    h->hflux_ready = false;  // the state or the step sequence changes
    int rc = flush_pending(h);
    return rc ? rc : op_energy_nodes(h);
}
int snac_gpu_calc_stresses(snac_gpu* h) {
    if (!h) return SNAC_GPU_EINVAL;
    h->hflux_ready = false;  // the state or the step sequence changes
    int rc = flush_pending(h);
    if (!rc) rc = op_calc_stresses(h);
    return rc ? rc : read_status(h);
}
int snac_gpu_loop_nodes_momentum(snac_gpu* h) {
    if (!h) return SNAC_GPU_EINVAL;
    h->hflux_ready = false;  // the state or the step sequence changes
    int rc = flush_pending(h);
    if (!rc) rc = op_loop_nodes(h);
    return rc ? rc : read_status(h);
}
int snac_gpu_loop_elements_momentum(snac_gpu* h) {
    if (!h) return SNAC_GPU_EINVAL;
    h->hflux_ready = false;  // the state or the step sequence changes
    int rc = flush_pending(h);
    if (!rc) rc = op_update_elements(h, h->time_step == 0);
    return rc ? rc : read_status(h);
}
int snac_gpu_sync(snac_gpu* h) {
    if (!h) return SNAC_GPU_EINVAL;
    h->hflux_ready = false;  // the state or the step sequence changes
    int rc = flush_pending(h);
    if (!rc) rc = op_sync_full(h);
    return rc ? rc : read_status(h);
}

int snac_gpu_upload(snac_gpu* h, const snac_state_view* v) {
    if (!h || !v) return SNAC_GPU_EINVAL;
    h->hflux_ready = false;  // the state or the step sequence changes
    if (int rc = flush_pending(h)) return rc;
    const long long nn = h->mesh.nn, nq = h->mesh.ne * NT;
    int rc;
    // every copy and repacking kernel is ordered on the handle's stream
    if (v->coord && (rc = node_in(h, h->pos[h->parity], v->coord, 0))) return rc;
    if (v->velocity && (rc = node_in(h, h->vel, v->velocity, 0))) return rc;
    if (v->temperature && (rc = node_in(h, h->pos[h->parity], v->temperature, 1))) return rc;
    if (v->stress) CK(cudaMemcpyAsync(h->stress, v->stress, nq * 6 * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    if (v->plastic_strain && h->eps_p)
        CK(cudaMemcpyAsync(h->eps_p, v->plastic_strain, nq * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    if (v->viscosity && h->visc)
        CK(cudaMemcpyAsync(h->visc, v->viscosity, nq * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    if (h->abi >= 2 && v->plastic_strain_tensor && h->pst)
        CK(cudaMemcpyAsync(h->pst, v->plastic_strain_tensor, nq * 6 * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));  // the caller may reuse its buffers on return
    (void)nn;
    return 0;
}

int snac_gpu_download(snac_gpu* h, const snac_state_view* v) {
    if (!h || !v) return SNAC_GPU_EINVAL;
    if (int rc = flush_pending(h)) return rc;
    const long long nq = h->mesh.ne * NT;
    int rc;
    if (v->coord && (rc = node_out(h, h->pos[h->parity], v->coord, 0))) return rc;
    if (v->velocity && (rc = node_out(h, h->vel, v->velocity, 0))) return rc;
    if (v->temperature && (rc = node_out(h, h->pos[h->parity], v->temperature, 1))) return rc;
    if (v->force && (rc = node_out(h, h->force, v->force, 0))) return rc;
    if (v->inertial_mass && (rc = node_out(h, h->force, v->inertial_mass, 1))) return rc;
    if (v->stress) CK(cudaMemcpyAsync(v->stress, h->stress, nq * 6 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    if (v->plastic_strain && h->eps_p)
        CK(cudaMemcpyAsync(v->plastic_strain, h->eps_p, nq * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    if (v->viscosity && h->visc)
        CK(cudaMemcpyAsync(v->viscosity, h->visc, nq * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    const bool want_pst = h->abi >= 2 && v->plastic_strain_tensor;
    if (want_pst && h->pst)
        CK(cudaMemcpyAsync(v->plastic_strain_tensor, h->pst, nq * 6 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (v->plastic_strain && !h->eps_p) memset(v->plastic_strain, 0, nq * sizeof(double));
    if (v->viscosity && !h->visc) memset(v->viscosity, 0, nq * sizeof(double));
    if (want_pst && !h->pst) memset(v->plastic_strain_tensor, 0, nq * 6 * sizeof(double));
    return 0;
}

// One step with the state in host memory, as snac_gpu_upload + snac_gpu_step(1)
// + snac_gpu_download, with the transfers overlapped slab by slab.  The mesh
// is cut along k (the slowest index of hexes and nodes) into `chunks` slabs
// of whole element blocks, and into as many node slabs of whole node blocks,
// node slab c ending below the first k-plane of element slab c + 1.  The step
// is a chain of stages that alternate between the two kinds of slab: the
// momentum step is stress update (hexes) -> force gather and node update
// (nodes) -> element update with the minimum length scale (hexes); models
// with temperature put heat flux (hexes) -> temperature update (nodes) in
// front.  A hex stage's slab reads the nodes of its k-planes and the next
// one, so it waits until the node stage before it has finished those nodes;
// a node stage's slab gathers from every hex of its planes and the planes
// below, so it waits until the hex stage before it has finished those hexes.
// A node slab only writes its own nodes, and by then no later slab of the
// earlier stages reads them.  The node state and the per-slab hex state are
// uploaded ahead on one stream, kernels run on the handle's stream, and each
// slab's results go back on a third stream once its last stage is done, so
// the host link carries both directions at once.  Every hex and node goes
// through the kernel bodies of the whole-mesh step and the reductions
// (max |v|, minimum length scale) are exact, so the result has the bits of
// the three calls.
// Queues the slab pipeline of one step (see snac_gpu_step_host) on the
// handle's stream and the two transfer streams; the handle's stream ends
// after every transfer of the step.
static int record_host_step(snac_gpu* h, const snac_state_view* in, const snac_state_view* out, int S) {
    int rc = 0;
    HostStep* q = h->hs;
    const Mesh& m = h->mesh;
    const long long ne = m.ne, nn = m.nn;
    // the stages of the step, alternating hex and node stages (snac_slab_plan.h)
    enum Stage { HEAT_FLUX, HEAT_NODES, STRESS, MOMENTUM_NODES, UPDATE };
    std::vector<Stage> stages;
    if (h->temperature) stages = {HEAT_FLUX, HEAT_NODES};
    stages.insert(stages.end(), {STRESS, MOMENTUM_NODES, UPDATE});
    const SlabPlan plan = plan_slabs(m.nx, m.ny, m.nz, S, (int)stages.size(), ELEM_PER_BLOCK, 128);
    const std::vector<long long>& E = plan.E;
    const std::vector<long long>& N = plan.N;
    const bool want_pst = out->plastic_strain_tensor != nullptr;
    const bool give_pst = in->plastic_strain_tensor != nullptr;
    const size_t D = sizeof(double);
    auto elems_in = [&](long long e0, long long e1) -> int {
        if (e1 <= e0) return 0;
        const long long a = e0 * NT, n = (e1 - e0) * NT;
        if (in->stress) CK(cudaMemcpyAsync(h->stress + a * 6, in->stress + a * 6, n * 6 * D, cudaMemcpyHostToDevice, q->in));
        if (in->plastic_strain && h->eps_p)
            CK(cudaMemcpyAsync(h->eps_p + a, in->plastic_strain + a, n * D, cudaMemcpyHostToDevice, q->in));
        if (in->viscosity && h->visc)
            CK(cudaMemcpyAsync(h->visc + a, in->viscosity + a, n * D, cudaMemcpyHostToDevice, q->in));
        if (give_pst && h->pst)
            CK(cudaMemcpyAsync(h->pst + a * 6, in->plastic_strain_tensor + a * 6, n * 6 * D, cudaMemcpyHostToDevice, q->in));
        return 0;
    };
    auto elems_out = [&](long long e0, long long e1) -> int {
        if (e1 <= e0) return 0;
        const long long a = e0 * NT, n = (e1 - e0) * NT;
        if (out->stress) CK(cudaMemcpyAsync(out->stress + a * 6, h->stress + a * 6, n * 6 * D, cudaMemcpyDeviceToHost, q->out));
        if (out->plastic_strain && h->eps_p)
            CK(cudaMemcpyAsync(out->plastic_strain + a, h->eps_p + a, n * D, cudaMemcpyDeviceToHost, q->out));
        if (out->viscosity && h->visc)
            CK(cudaMemcpyAsync(out->viscosity + a, h->visc + a, n * D, cudaMemcpyDeviceToHost, q->out));
        if (want_pst && h->pst)
            CK(cudaMemcpyAsync(out->plastic_strain_tensor + a * 6, h->pst + a * 6, n * 6 * D, cudaMemcpyDeviceToHost, q->out));
        return 0;
    };

    const int p = h->parity;
    const Fields F0 = fields_at(h, p);      // this step: coordinates in pos[p], moved into pos[p ^ 1]
    const Fields F1 = fields_at(h, p ^ 1);  // the element update reads the moved coordinates
    double* const si = q->stage_in;         // [coordinates | velocities | temperatures]
    double* const so = q->stage_out;
    CK(cudaEventRecord(q->start, h->stream));  // after anything the handle ran before
    CK(cudaStreamWaitEvent(q->in, q->start, 0));
    CK(cudaStreamWaitEvent(q->out, q->start, 0));
    // Uploads, all queued at once: the node rows the first two hex slabs
    // read, those two slabs, the other node rows, then the other hex slabs;
    // the first downloads wait for the second slab, so it arrives early.
    const bool node_in = in->coord || in->velocity || in->temperature;
    const long long n_head = plan.n_head;
    auto nodes_up = [&](long long a, long long b) -> int {
        if (b <= a) return 0;
        if (in->coord) CK(cudaMemcpyAsync(si + a * 3, in->coord + a * 3, (b - a) * 3 * D, cudaMemcpyHostToDevice, q->in));
        if (in->velocity)
            CK(cudaMemcpyAsync(si + (nn + a) * 3, in->velocity + a * 3, (b - a) * 3 * D, cudaMemcpyHostToDevice, q->in));
        if (in->temperature)
            CK(cudaMemcpyAsync(si + nn * 6 + a, in->temperature + a, (b - a) * D, cudaMemcpyHostToDevice, q->in));
        return 0;
    };
    auto nodes_unpack = [&](long long a, long long b) -> int {
        if (b <= a || !node_in) return 0;
        k_unpack_node_state<<<(unsigned)((b - a + 255) / 256), 256, 0, h->stream>>>(
            h->pos[p] + a, in->coord ? si + a * 3 : nullptr, in->temperature ? si + nn * 6 + a : nullptr, h->vel + a,
            in->velocity ? si + (nn + a) * 3 : nullptr, b - a);
        h->launches++;
        return launch_check_named(h, "k_unpack_node_state");
    };
    if ((rc = nodes_up(0, n_head))) return rc;
    CK(cudaEventRecord(q->nodes_in, q->in));
    for (int c = 0; c < S; c++) {
        if (c == std::min(2, S)) {
            if ((rc = nodes_up(n_head, nn))) return rc;
            CK(cudaEventRecord(q->nodes_rest, q->in));
        }
        if ((rc = elems_in(E[c], E[c + 1]))) return rc;
        CK(cudaEventRecord(q->ev_in[c], q->in));
    }
    if (S <= 2) {  // (then the first two slabs read every node: nothing left)
        if ((rc = nodes_up(n_head, nn))) return rc;
        CK(cudaEventRecord(q->nodes_rest, q->in));
    }
    if ((rc = op_begin(h))) return rc;  // timeStep++, currentTime += dt
    CK(cudaStreamWaitEvent(h->stream, q->nodes_in, 0));
    if ((rc = nodes_unpack(0, n_head))) return rc;

    const bool node_rows = out->coord || out->velocity || out->temperature;
    int kernels = 0;
    for (const SlabOp& o : plan.ops) {
        if (o.kind == SlabOp::UNPACK_REST) {  // nodes [n_head, nn), before hex slab 2 of the first stage
            CK(cudaStreamWaitEvent(h->stream, q->nodes_rest, 0));
            if ((rc = nodes_unpack(n_head, nn))) return rc;
            continue;
        }
        if (o.kind == SlabOp::NODES_BACK) {  // node slabs up to this one are packed
            const long long a = o.a, n = o.b - o.a;
            if (n > 0 && out->coord)
                CK(cudaMemcpyAsync(out->coord + a * 3, so + a * 3, n * 3 * D, cudaMemcpyDeviceToHost, q->out));
            if (n > 0 && out->velocity)
                CK(cudaMemcpyAsync(out->velocity + a * 3, so + nn * 3 + a * 3, n * 3 * D, cudaMemcpyDeviceToHost, q->out));
            if (n > 0 && out->temperature)
                CK(cudaMemcpyAsync(out->temperature + a, so + nn * 6 + a, n * D, cudaMemcpyDeviceToHost, q->out));
            continue;
        }
        if (o.kind == SlabOp::HEXES_BACK) {
            if ((rc = elems_out(E[o.slab], E[o.slab + 1]))) return rc;
            continue;
        }
        const int s = o.stage, i = o.slab;
        if (s == 0) CK(cudaStreamWaitEvent(h->stream, q->ev_in[i], 0));
        const int b0 = (int)(E[i] / ELEM_PER_BLOCK), b1 = (int)((E[i + 1] + ELEM_PER_BLOCK - 1) / ELEM_PER_BLOCK);
        const int n0 = (int)(N[i] / 128), n1 = (int)((N[i + 1] + 127) / 128);
        switch (stages[s]) {
            case HEAT_FLUX: rc = op_heat_flux_slab(h, F0, b0, b1); break;
            case HEAT_NODES: rc = op_heat_nodes_slab(h, F0, n0, n1); break;
            case STRESS: rc = op_calc_stresses_slab(h, F0, b0, b1); break;
            case MOMENTUM_NODES: rc = op_loop_nodes_slab(h, F0, n0, n1); break;
            case UPDATE: rc = op_update_elements_slab(h, F1, b0, b1); break;
        }
        if (rc) return rc;
        kernels++;
        if (stages[s] == MOMENTUM_NODES && N[i + 1] > N[i] && node_rows) {
            const long long a = N[i], n = N[i + 1] - N[i];
            k_pack_node_state<<<(unsigned)((n + 255) / 256), 256, 0, h->stream>>>(
                h->pos[p ^ 1] + a, out->coord ? so + a * 3 : nullptr, out->temperature ? so + nn * 6 + a : nullptr,
                h->vel + a, out->velocity ? so + nn * 3 + a * 3 : nullptr, n);
            h->launches++;
            if ((rc = launch_check_named(h, "k_pack_node_state"))) return rc;
        }
        if (stages[s] == UPDATE) {  // the slab's downloads (the plan's next ops) wait for this
            CK(cudaEventRecord(q->ev_elems[i], h->stream));
            CK(cudaStreamWaitEvent(q->out, q->ev_elems[i], 0));
        }
    }
    if (kernels != (int)stages.size() * S)  // the plan always finishes every slab of every stage
        return set_err(h, SNAC_GPU_ESTATE, -1, "snac_gpu_step_host: slab plan has %d of %d slab kernels", kernels,
                       (int)stages.size() * S);
    (void)ne;
    if ((rc = op_sync(h))) return rc;  // Sync: the next dt from this step's reductions
    CK(cudaEventRecord(q->done, q->out));
    CK(cudaStreamWaitEvent(h->stream, q->done, 0));
    return 0;
}

int snac_gpu_step_host(snac_gpu* h, const snac_state_view* in, const snac_state_view* out, int chunks) {
    if (!h || !in || !out) return SNAC_GPU_EINVAL;
    if (chunks < 0 || chunks > STEP_HOST_MAX_CHUNKS)
        return set_err(h, SNAC_GPU_EINVAL, -1, "snac_gpu_step_host: chunks = %d, allowed 0 (default) to %d", chunks,
                       STEP_HOST_MAX_CHUNKS);
    if (!h->zero_done) return set_err(h, SNAC_GPU_ESTATE, -1, "snac_gpu_time_step_zero must come first");
    // Topography diffusion (a wavefront over the whole top surface), dump
    // files, kernel timing and node fields the step does not move take the
    // three calls.
    const bool slabs = !topo_on(h->cfg) && !h->out && h->own_stream && !h->prof && !out->force && !out->inertial_mass;
    if (!slabs) {
        int rc = snac_gpu_upload(h, in);
        if (!rc) rc = snac_gpu_step(h, 1);
        if (!rc) rc = snac_gpu_download(h, out);
        return rc;
    }
    int rc = ensure_host_step(h);
    if (rc) return rc;
    HostStep* q = h->hs;
    h->hflux_ready = false;  // this step forms its own heat flux
    if ((rc = flush_pending(h))) return rc;
    // the caller's views as this handle reads them (a version-1 view has no
    // plastic-strain tensor)
    snac_state_view vi{}, vo{};
    const size_t vbytes = h->abi >= 2 ? sizeof(snac_state_view) : offsetof(snac_state_view, plastic_strain_tensor);
    memcpy(&vi, in, vbytes);
    memcpy(&vo, out, vbytes);
    // default: one slab per 6 MiB of stresses (the bulk of the transfers),
    // 1 to 16 slabs; smaller slabs cost more in per-slab latency than they
    // save in pipeline fill
    const long long stress_bytes = h->mesh.ne * NT * 6 * (long long)sizeof(double);
    const int S = chunks ? chunks : (int)std::max(1LL, std::min(16LL, (stress_bytes + (3LL << 20)) / (6LL << 20)));
    {
        // every return below waits for this call's copies first: the caller
        // may release its host buffers once the call has returned
        struct Drain {
            HostStep* q;
            cudaStream_t s;
            ~Drain() {
                cudaStreamSynchronize(q->in);
                cudaStreamSynchronize(q->out);
                cudaStreamSynchronize(s);
            }
        } drain{q, h->stream};
        if ((rc = record_host_step(h, &vi, &vo, S))) return rc;
    }
    h->parity ^= 1;
    h->pending = false;
    CK(cudaStreamSynchronize(h->stream));
    if ((rc = read_status(h))) return rc;
    const long long nq = h->mesh.ne * NT;
    if (out->plastic_strain && !h->eps_p) memset(out->plastic_strain, 0, nq * sizeof(double));
    if (out->viscosity && !h->visc) memset(out->viscosity, 0, nq * sizeof(double));
    if (vo.plastic_strain_tensor && !h->pst) memset(vo.plastic_strain_tensor, 0, nq * 6 * sizeof(double));
    return 0;
}

int snac_gpu_scalars(snac_gpu* h, snac_scalars* out) {
    if (!h || !out) return SNAC_GPU_EINVAL;
    DevScalars s;
    CK(cudaMemcpyAsync(&s, h->sc, sizeof s, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    out->dt = s.dt;
    out->min_length_scale = s.min_length_scale;
    out->vmax = s.vmax;
    out->speed_of_sound = s.speed_of_sound;
    out->time_step = s.time_step;
    out->current_time = s.current_time;
    return 0;
}

int snac_gpu_set_dt(snac_gpu* h, double dt) {
    if (!h) return SNAC_GPU_EINVAL;
    CK(cudaMemcpyAsync(&h->sc->dt, &dt, sizeof dt, cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return 0;
}

const char* snac_gpu_last_error(const snac_gpu* h) { return h ? h->err : "null handle"; }
long long snac_gpu_error_index(const snac_gpu* h) { return h ? h->err_index : -1; }
int snac_gpu_sizes(const snac_gpu* h, long long* ne, long long* nn) {
    if (!h) return SNAC_GPU_EINVAL;
    if (ne) *ne = h->mesh.ne;
    if (nn) *nn = h->mesh.nn;
    return 0;
}
long long snac_gpu_launch_count(const snac_gpu* h) { return h ? h->launches : 0; }

int snac_gpu_device_bytes(const snac_gpu* h, long long* bytes) {
    if (!h || !bytes) return SNAC_GPU_EINVAL;
    *bytes = h->alloc_bytes;
    return 0;
}

int snac_gpu_profile_step(snac_gpu* h, snac_kernel_time* out, int max) {
    if (!h || !out || max < 1) return SNAC_GPU_EINVAL;
    if (!h->zero_done) return set_err(h, SNAC_GPU_ESTATE, -1, "snac_gpu_time_step_zero must come first");
    for (auto& e : h->prof_ev) CK(cudaEventCreate(&e));
    h->prof = out;
    h->prof_n = 0;
    h->prof_max = max;
    CK(cudaEventRecord(h->prof_ev[0], h->stream));
    bool fused = h->pending;
    int rc = record_step(h, fused);
    h->prof = nullptr;
    if (!rc) {
        h->parity ^= 0;  // record_step already flipped the parity in the node loop
        h->pending = true;
        h->hflux_ready = h->temperature;  // the step's last kernel formed the next heat flux
        CK(cudaStreamSynchronize(h->stream));
        for (int i = 0; i < h->prof_n; i++) {
            float ms = 0;
            cudaEventElapsedTime(&ms, h->prof_ev[i], h->prof_ev[i + 1]);
            out[i].ms = ms;
        }
    }
    for (auto& e : h->prof_ev) cudaEventDestroy(e);
    if (rc) return rc;
    rc = read_status(h);
    return rc ? rc : h->prof_n;
}
void* snac_gpu_stream(snac_gpu* h) { return h ? (void*)h->stream : nullptr; }

}  // extern "C"

// ======================================================================================
// Batched ensembles: every model keeps its own buffers; the batch adds per-model
// descriptors (one table per coordinate parity) and tile lists, and launches
// each kernel type once per step over all models.
// ======================================================================================
struct snac_gpu_batch {
    std::vector<snac_gpu*> models;
    cudaStream_t stream = nullptr;
    int n = 0;
    int n_sm = 148;
    ModelDesc* desc[2] = {nullptr, nullptr};  // [parity]
    int2* tiles = nullptr;
    size_t tiles_cap = 0;
    struct List {
        long long off = 0;
        int n = 0;
    };
    List elem_all, elem_temp, node_all, node_temp, minls_all;
    List elem_cls[NCLASS];  // element tiles grouped by rheology class (plugin, temperature)
    bool any_temp = false;
    snac_batch_tuning tune{128, 128, 0, 0, 8, 0, 1};
    bool tiles_dirty = true;
    cudaGraphExec_t graph[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};  // [multi-step chunk][start parity]
    int graph_kernels[2] = {0, 0};
    ModelStatus* d_status = nullptr;
    std::vector<ModelStatus> h_status;
    int parity = 0;
    long long launches = 0;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    char err[512] = {0};
    int err_model = -1;
};

namespace {

int bset_err(snac_gpu_batch* b, int code, int model, const char* fmt, ...) {
    if (!b) return code;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(b->err, sizeof b->err, fmt, ap);
    va_end(ap);
    b->err_model = model;
    return code;
}

#define BCK(call)                                                                                        \
    do {                                                                                                 \
        cudaError_t e_ = (call);                                                                         \
        if (e_ != cudaSuccess) return bset_err(b, SNAC_GPU_ECUDA, -1, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

void drop_graphs(snac_gpu_batch* b) {
    for (auto& gc : b->graph)
        for (auto& g : gc)
            if (g) {
                cudaGraphExecDestroy(g);
                g = nullptr;
            }
}

int build_desc(snac_gpu_batch* b) {
    std::vector<ModelDesc> d(b->n);
    for (int p = 0; p < 2; p++) {
        for (int i = 0; i < b->n; i++) {
            const snac_gpu* h = b->models[i];
            d[i].m = h->mesh;
            d[i].F = fields_at(h, p);
            d[i].cfg = h->cfg;
            d[i].cfg.time_step_zero = 0;
            d[i].wave_speed = h->wave_speed;
        }
        BCK(cudaMemcpyAsync(b->desc[p], d.data(), b->n * sizeof(ModelDesc), cudaMemcpyHostToDevice, b->stream));
        BCK(cudaStreamSynchronize(b->stream));
    }
    return 0;
}

// Tile lists for the current launch shape.  Order 0 puts the largest models
// first (longest-processing-time first), so the last wave of a launch holds
// the small tiles.
int build_tiles(snac_gpu_batch* b) {
    std::vector<int> order(b->n);
    for (int i = 0; i < b->n; i++) order[i] = i;
    if (b->tune.order == 0)
        std::stable_sort(order.begin(), order.end(),
                         [&](int x, int y) { return b->models[x]->mesh.ne > b->models[y]->mesh.ne; });
    std::vector<int2> t;
    auto add = [&](snac_gpu_batch::List& L, bool temp_only, int kind) {
        L.off = (long long)t.size();
        for (int i : order) {
            const snac_gpu* h = b->models[i];
            if (temp_only && !h->temperature) continue;
            long long nb = kind == 0   ? (long long)elem_blocks(h->mesh)
                           : kind == 1 ? (h->mesh.nn + b->tune.node_threads - 1) / b->tune.node_threads
                                       : (h->mesh.ne + b->tune.minls_threads - 1) / b->tune.minls_threads;
            for (long long k = 0; k < nb; k++) t.push_back(make_int2(i, (int)k));
        }
        L.n = (int)((long long)t.size() - L.off);
    };
    add(b->elem_all, false, 0);
    add(b->elem_temp, true, 0);
    for (int c = 0; c < NCLASS; c++) {  // the same element tiles, class by class
        snac_gpu_batch::List& L = b->elem_cls[c];
        L.off = (long long)t.size();
        for (int i : order) {
            const snac_gpu* h = b->models[i];
            if (plugin_slot(h->constitutive) * 2 + (h->temperature ? 1 : 0) != c) continue;
            const long long nb = (long long)elem_blocks(h->mesh);
            for (long long k = 0; k < nb; k++) t.push_back(make_int2(i, (int)k));
        }
        L.n = (int)((long long)t.size() - L.off);
    }
    add(b->node_all, false, 1);
    add(b->node_temp, true, 1);
    add(b->minls_all, false, 2);
    if (t.size() > (size_t)0x7fffffff) return bset_err(b, SNAC_GPU_EINVAL, -1, "too many tiles in one batch");
    if (t.size() > b->tiles_cap) {
        if (b->tiles) cudaFree(b->tiles);
        b->tiles = nullptr;
        b->tiles_cap = 0;
        cudaError_t e = cudaMalloc((void**)&b->tiles, t.size() * sizeof(int2));
        if (e != cudaSuccess) return bset_err(b, SNAC_GPU_ENOMEM, -1, "cudaMalloc(tiles): %s", cudaGetErrorString(e));
        b->tiles_cap = t.size();
    }
    BCK(cudaMemcpyAsync(b->tiles, t.data(), t.size() * sizeof(int2), cudaMemcpyHostToDevice, b->stream));
    BCK(cudaStreamSynchronize(b->stream));
    drop_graphs(b);
    b->tiles_dirty = false;
    return 0;
}

unsigned tile_grid(const snac_gpu_batch* b, int ntiles, int per_sm) {
    long long g = ntiles;
    if (per_sm > 0) g = std::min<long long>(g, (long long)per_sm * b->n_sm);
    return (unsigned)std::max<long long>(g, 1);
}

int bcheck_launch(snac_gpu_batch* b, const char* name) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return bset_err(b, SNAC_GPU_ECUDA, -1, "%s launch: %s", name, cudaGetErrorString(e));
    b->launches++;
    return 0;
}

template <int OP>
int blaunch_elem(snac_gpu_batch* b, const ModelDesc* D, const snac_gpu_batch::List& L) {
    if (L.n == 0) return 0;
    kb_elements<OP><<<tile_grid(b, L.n, b->tune.elem_blocks_per_sm), ELEM_WARPS * 32, 0, b->stream>>>(D, b->tiles + L.off, L.n);
    return bcheck_launch(b, "kb_elements");
}

template <int OP>
int blaunch_nodes(snac_gpu_batch* b, const ModelDesc* D, const snac_gpu_batch::List& L, int threads) {
    if (L.n == 0) return 0;
    kb_nodes<OP><<<tile_grid(b, L.n, b->tune.node_blocks_per_sm), threads, 0, b->stream>>>(D, b->tiles + L.off, L.n);
    return bcheck_launch(b, "kb_nodes");
}

template <int OP, int P, int TEMP>
int blaunch_elem_c(snac_gpu_batch* b, const ModelDesc* D, const snac_gpu_batch::List& L) {
    if (L.n == 0) return 0;
    kb_elements_c<OP, P, TEMP><<<tile_grid(b, L.n, b->tune.elem_blocks_per_sm), ELEM_WARPS * 32, 0, b->stream>>>(
        D, b->tiles + L.off, L.n);
    return bcheck_launch(b, "kb_elements_c");
}

// one launch per rheology class present; temp_only skips the classes without temperature
template <int OP>
int blaunch_elem_classes(snac_gpu_batch* b, const ModelDesc* D, bool temp_only) {
    int rc = 0;
    const auto& C = b->elem_cls;
    if (!temp_only) {
        if (!rc) rc = blaunch_elem_c<OP, SNAC_RHEOLOGY_ELASTIC, 0>(b, D, C[0]);
        if (!rc) rc = blaunch_elem_c<OP, SNAC_RHEOLOGY_PLASTIC, 0>(b, D, C[2]);
    }
    if (!rc) rc = blaunch_elem_c<OP, SNAC_RHEOLOGY_ELASTIC, 1>(b, D, C[1]);
    if (!rc) rc = blaunch_elem_c<OP, SNAC_RHEOLOGY_PLASTIC, 1>(b, D, C[3]);
    if (!rc) rc = blaunch_elem_c<OP, SNAC_RHEOLOGY_VISCOPLASTIC, 1>(b, D, C[5]);
    if (!rc) rc = blaunch_elem_c<OP, SNAC_RHEOLOGY_MAXWELL, 1>(b, D, C[7]);
    return rc;  // classes 4 and 6 (visco-plastic / Maxwell without temperature) cannot be created
}

// one step of every model, in the order of record_step
int record_batch_step(snac_gpu_batch* b, bool fused, int parity) {
    const ModelDesc* D = b->desc[parity];
    const unsigned mb = (unsigned)((b->n + 127) / 128);
    int rc;
    const bool by_class = b->tune.split_classes != 0;
    if (fused) {
        if ((rc = by_class ? blaunch_elem_classes<BOP_FUSED>(b, D, false) : blaunch_elem<BOP_FUSED>(b, D, b->elem_all)))
            return rc;
    } else {
        kb_begin_step<<<mb, 128, 0, b->stream>>>(D, b->n);
        if ((rc = bcheck_launch(b, "kb_begin_step"))) return rc;
        if ((rc = by_class ? blaunch_elem_classes<BOP_HEAT_FLUX>(b, D, true)
                           : blaunch_elem<BOP_HEAT_FLUX>(b, D, b->elem_temp)))
            return rc;
    }
    if ((rc = blaunch_nodes<BOP_HEAT_NODES>(b, D, b->node_temp, b->tune.node_threads))) return rc;
    // temperature models: after the energy hooks, the pending element update
    // fused with the stress update (fused step) or the stress update alone
    if (fused)
        rc = by_class ? blaunch_elem_classes<BOP_FUSED_STRESS>(b, D, true)
                      : blaunch_elem<BOP_FUSED_STRESS>(b, D, b->elem_temp);
    else
        rc = by_class ? blaunch_elem_classes<BOP_STRESS>(b, D, false) : blaunch_elem<BOP_STRESS>(b, D, b->elem_all);
    if (rc) return rc;
    if ((rc = blaunch_nodes<BOP_LOOP_NODES>(b, D, b->node_all, b->tune.node_threads))) return rc;
    // the node loop wrote the new coordinates into the other buffer
    const ModelDesc* Dn = b->desc[parity ^ 1];
    if ((rc = blaunch_nodes<BOP_MINLS>(b, Dn, b->minls_all, b->tune.minls_threads))) return rc;
    kb_sync<<<mb, 128, 0, b->stream>>>(D, b->n);
    return bcheck_launch(b, "kb_sync");
}

// models of a batch step together: same parity, all past step zero, and
// either all or none with a deferred element update (a model whose state was
// downloaded on its own has had its update applied; the others are flushed too)
int batch_prepare(snac_gpu_batch* b, bool* fused) {
    int npending = 0;
    for (int i = 0; i < b->n; i++) {
        snac_gpu* h = b->models[i];
        if (!h->zero_done) return bset_err(b, SNAC_GPU_ESTATE, i, "model %d: time step zero must come first", i);
        if (h->parity != b->models[0]->parity)
            return bset_err(b, SNAC_GPU_ESTATE, i, "model %d was stepped on its own: the models are out of step", i);
        npending += h->pending ? 1 : 0;
    }
    if (npending != 0 && npending != b->n) {
        for (int i = 0; i < b->n; i++) {
            int rc = flush_pending(b->models[i]);
            if (rc) return bset_err(b, rc, i, "model %d: %s", i, b->models[i]->err);
        }
        npending = 0;
    }
    *fused = npending == b->n;
    b->parity = b->models[0]->parity;
    if (b->tiles_dirty) return build_tiles(b);
    return 0;
}

// launches nsteps batched steps (no status read)
int batch_run(snac_gpu_batch* b, int nsteps) {
    bool fused;
    int rc;
    if ((rc = batch_prepare(b, &fused))) return rc;
    int s = 0;
    if (!fused && nsteps > 0) {
        if ((rc = record_batch_step(b, false, b->parity))) return rc;
        b->parity ^= 1;
        s = 1;
    }
    const int S = b->tune.steps_per_graph;
    while (s < nsteps) {
        const int chunk = (S > 1 && nsteps - s >= S) ? 1 : 0;
        const int k = chunk ? S : 1;
        cudaGraphExec_t& ge = b->graph[chunk][b->parity];
        if (!ge) {
            cudaGraph_t g;
            long long l0 = b->launches;
            BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
            int rc2 = 0;
            for (int j = 0; j < k && !rc2; j++) rc2 = record_batch_step(b, true, b->parity ^ (j & 1));
            cudaError_t e = cudaStreamEndCapture(b->stream, &g);
            if (rc2) return rc2;
            if (e != cudaSuccess) return bset_err(b, SNAC_GPU_ECUDA, -1, "graph capture: %s", cudaGetErrorString(e));
            e = cudaGraphInstantiate(&ge, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) return bset_err(b, SNAC_GPU_ECUDA, -1, "graph instantiate: %s", cudaGetErrorString(e));
            b->graph_kernels[chunk] = (int)(b->launches - l0);
            b->launches = l0;
        }
        BCK(cudaGraphLaunch(ge, b->stream));
        b->launches += b->graph_kernels[chunk];
        s += k;
        b->parity ^= (k & 1);
    }
    for (snac_gpu* h : b->models) {
        h->time_step += nsteps;
        h->parity = b->parity;
        if (nsteps > 0) h->pending = true;
        h->hflux_ready = false;  // the batched step forms each step's heat flux itself
    }
    return 0;
}

// the same steps model by model, each with its own step graph
int batch_run_each(snac_gpu_batch* b, int nsteps) {
    bool fused;
    int rc;
    if ((rc = batch_prepare(b, &fused))) return rc;
    for (int s = 0; s < nsteps; s++)
        for (int i = 0; i < b->n; i++) {
            snac_gpu* h = b->models[i];
            long long l0 = h->launches;
            if ((rc = launch_step(h))) return bset_err(b, rc, i, "model %d: %s", i, h->err);
            b->launches += h->launches - l0;
        }
    b->parity = b->models[0]->parity;
    return 0;
}

int batch_status(snac_gpu_batch* b) {
    kb_status<<<(unsigned)((b->n + 127) / 128), 128, 0, b->stream>>>(b->desc[0], b->n, b->d_status);
    BCK(cudaGetLastError());
    BCK(cudaMemcpyAsync(b->h_status.data(), b->d_status, b->n * sizeof(ModelStatus), cudaMemcpyDeviceToHost, b->stream));
    BCK(cudaStreamSynchronize(b->stream));
    for (int i = 0; i < b->n; i++) {
        if (b->h_status[i].status) {
            int rc = read_status(b->models[i]);  // the model's own message
            return bset_err(b, rc ? rc : b->h_status[i].status, i, "model %d: %s", i, b->models[i]->err);
        }
    }
    return 0;
}

}  // namespace

extern "C" {

int snac_gpu_batch_create(const snac_gpu_desc* descs, int n_models, snac_gpu_batch** out) {
    if (!out) return SNAC_GPU_EINVAL;
    *out = nullptr;
    if (!descs || n_models < 1) return SNAC_GPU_EINVAL;
    snac_gpu_batch* b = new (std::nothrow) snac_gpu_batch();
    if (!b) return SNAC_GPU_ENOMEM;
    *out = b;
    int dev = 0;
    BCK(cudaGetDevice(&dev));
    BCK(cudaDeviceGetAttribute(&b->n_sm, cudaDevAttrMultiProcessorCount, dev));
    BCK(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    BCK(cudaEventCreate(&b->ev[0]));
    BCK(cudaEventCreate(&b->ev[1]));
    b->n = n_models;
    b->models.assign(n_models, nullptr);
    for (int i = 0; i < n_models; i++) {
        int rc = create_model(&descs[i], &b->models[i], b->stream);
        if (rc) {
            const char* msg = b->models[i] ? b->models[i]->err : "invalid descriptor";
            return bset_err(b, rc, i, "model %d: %s", i, msg[0] ? msg : "invalid descriptor");
        }
        if (b->models[i]->dp)  // the batched kernels have no Drucker-Prager instances
            return bset_err(b, SNAC_GPU_ENOTSUP, i, "model %d: Drucker-Prager phases are not batched", i);
        b->any_temp = b->any_temp || b->models[i]->temperature;
        if (topo_on(b->models[i]->cfg))
            return bset_err(b, SNAC_GPU_ENOTSUP, i, "model %d: topography diffusion is not batched", i);
    }
    cudaError_t e = cudaMalloc((void**)&b->desc[0], n_models * sizeof(ModelDesc));
    if (e == cudaSuccess) e = cudaMalloc((void**)&b->desc[1], n_models * sizeof(ModelDesc));
    if (e == cudaSuccess) e = cudaMalloc((void**)&b->d_status, n_models * sizeof(ModelStatus));
    if (e != cudaSuccess) return bset_err(b, SNAC_GPU_ENOMEM, -1, "cudaMalloc: %s", cudaGetErrorString(e));
    b->h_status.resize(n_models);
    return build_desc(b);
}

void snac_gpu_batch_destroy(snac_gpu_batch* b) {
    if (!b) return;
    if (b->stream) cudaStreamSynchronize(b->stream);
    drop_graphs(b);
    for (snac_gpu* h : b->models)
        if (h) snac_gpu_destroy(h);
    void* bufs[] = {b->desc[0], b->desc[1], b->tiles, b->d_status};
    for (void* p : bufs)
        if (p) cudaFree(p);
    for (cudaEvent_t ev : b->ev)
        if (ev) cudaEventDestroy(ev);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

int snac_gpu_batch_time_step_zero(snac_gpu_batch* b) {
    if (!b) return SNAC_GPU_EINVAL;
    for (int i = 0; i < b->n; i++) {
        int rc = snac_gpu_time_step_zero(b->models[i]);
        if (rc) return bset_err(b, rc, i, "model %d: %s", i, b->models[i]->err);
    }
    return 0;
}

int snac_gpu_batch_step(snac_gpu_batch* b, int nsteps) {
    if (!b || nsteps < 0) return SNAC_GPU_EINVAL;
    int rc = batch_run(b, nsteps);
    return rc ? rc : batch_status(b);
}

int snac_gpu_batch_step_each(snac_gpu_batch* b, int nsteps) {
    if (!b || nsteps < 0) return SNAC_GPU_EINVAL;
    int rc = batch_run_each(b, nsteps);
    return rc ? rc : batch_status(b);
}

int snac_gpu_batch_time_steps(snac_gpu_batch* b, int nsteps, int each, double* ms) {
    if (!b || nsteps < 0 || !ms) return SNAC_GPU_EINVAL;
    bool fused;
    int rc = batch_prepare(b, &fused);  // tile lists and flushes outside the timed region
    if (rc) return rc;
    BCK(cudaEventRecord(b->ev[0], b->stream));
    rc = each ? batch_run_each(b, nsteps) : batch_run(b, nsteps);
    if (rc) return rc;
    BCK(cudaEventRecord(b->ev[1], b->stream));
    if ((rc = batch_status(b))) return rc;
    float t = 0.0f;
    BCK(cudaEventElapsedTime(&t, b->ev[0], b->ev[1]));
    *ms = t;
    return 0;
}

snac_gpu* snac_gpu_batch_model(snac_gpu_batch* b, int i) {
    if (!b || i < 0 || i >= b->n) return nullptr;
    return b->models[i];
}

int snac_gpu_batch_size(const snac_gpu_batch* b) { return b ? b->n : 0; }

int snac_gpu_batch_get_tuning(const snac_gpu_batch* b, snac_batch_tuning* out) {
    if (!b || !out) return SNAC_GPU_EINVAL;
    *out = b->tune;
    return 0;
}

int snac_gpu_batch_set_tuning(snac_gpu_batch* b, const snac_batch_tuning* t) {
    if (!b || !t) return SNAC_GPU_EINVAL;
    auto threads_ok = [](int x) { return x >= 32 && x <= 256 && x % 32 == 0; };
    if (!threads_ok(t->node_threads) || !threads_ok(t->minls_threads) || t->elem_blocks_per_sm < 0 ||
        t->elem_blocks_per_sm > 32 || t->node_blocks_per_sm < 0 || t->node_blocks_per_sm > 32 ||
        t->steps_per_graph < 1 || t->steps_per_graph > 256 || (t->order != 0 && t->order != 1) ||
        (t->split_classes != 0 && t->split_classes != 1))
        return bset_err(b, SNAC_GPU_EINVAL, -1, "launch shape out of range");
    const snac_batch_tuning o = b->tune;
    b->tune = *t;
    if (o.node_threads != t->node_threads || o.minls_threads != t->minls_threads || o.order != t->order)
        b->tiles_dirty = true;
    else if (o.elem_blocks_per_sm != t->elem_blocks_per_sm || o.node_blocks_per_sm != t->node_blocks_per_sm ||
             o.steps_per_graph != t->steps_per_graph || o.split_classes != t->split_classes)
        drop_graphs(b);
    return 0;
}

const char* snac_gpu_batch_last_error(const snac_gpu_batch* b) { return b ? b->err : "null batch"; }
int snac_gpu_batch_error_model(const snac_gpu_batch* b) { return b ? b->err_model : -1; }
long long snac_gpu_batch_launch_count(const snac_gpu_batch* b) { return b ? b->launches : 0; }
void* snac_gpu_batch_stream(snac_gpu_batch* b) { return b ? (void*)b->stream : nullptr; }

}  // extern "C"

// ======================================================================================
// Node-field download without any allocation: the staging lives in a
// file-scope device array instead of the handle's lazily allocated buffer.
// ======================================================================================
namespace {

constexpr long long NOALLOC_MAX_NODES = 262144;  // 262,144 nodes x 3 doubles = 6 MiB

// every element the call copies out was written by k_pack_nodes earlier in
// the same call, so no part of it has to start at zero
__device__ __align__(256) double g_noalloc_stage[NOALLOC_MAX_NODES * 3];

constexpr int NOALLOC_MAX_DEVICES = 64;
void* g_noalloc_addr[NOALLOC_MAX_DEVICES] = {nullptr};
std::mutex g_noalloc_lock;  // held for a whole call: one staging array per device

int noalloc_node_out(snac_gpu* h, double* stage, const double4* src, double* dst, int what) {
    const long long nn = h->mesh.nn;
    k_pack_nodes<<<(unsigned)((nn + 255) / 256), 256, 0, h->stream>>>(src, stage, nn, what);
    h->launches++;
    int rc = launch_check_named(h, "k_pack_nodes");
    if (rc) return rc;
    CK(cudaMemcpyAsync(dst, stage, nn * (what == 0 ? 3 : 1) * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    return 0;
}

}  // namespace

extern "C" int snac_gpu_download_nodes_noalloc(snac_gpu* h, double* coord, double* velocity, double* temperature) {
    if (!h) return SNAC_GPU_EINVAL;
    if (h->mesh.nn > NOALLOC_MAX_NODES)
        return set_err(h, SNAC_GPU_EINVAL, -1,
                       "snac_gpu_download_nodes_noalloc: the model has %lld nodes, the static staging holds at most %lld",
                       h->mesh.nn, NOALLOC_MAX_NODES);
    int dev = -1;
    CK(cudaGetDevice(&dev));
    cudaPointerAttributes pa;
    CK(cudaPointerGetAttributes(&pa, h->vel));
    if (pa.device != dev)
        return set_err(h, SNAC_GPU_EINVAL, -1,
                       "snac_gpu_download_nodes_noalloc: the handle lives on device %d, device %d is current", pa.device, dev);
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return set_err(h, SNAC_GPU_EINVAL, -1, "device index %d out of range", dev);
    std::lock_guard<std::mutex> guard(g_noalloc_lock);
    if (!g_noalloc_addr[dev]) {  // once per device, with that device current
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_stage);
        if (e != cudaSuccess || !p)
            return set_err(h, SNAC_GPU_ECUDA, -1, "cudaGetSymbolAddress(staging): %s", cudaGetErrorString(e));
        g_noalloc_addr[dev] = p;
    }
    double* stage = static_cast<double*>(g_noalloc_addr[dev]);
    int rc;
    if ((rc = flush_pending(h))) return rc;  // does not touch the staging
    if (coord) rc = noalloc_node_out(h, stage, h->pos[h->parity], coord, 0);
    if (!rc && velocity) rc = noalloc_node_out(h, stage, h->vel, velocity, 0);
    if (!rc && temperature) rc = noalloc_node_out(h, stage, h->pos[h->parity], temperature, 1);
    // Whatever happened above, this call's packs and copies are finished
    // before the lock is released, so the next caller finds the staging free
    // (and, on success, the host arrays are filled).
    const cudaError_t se = cudaStreamSynchronize(h->stream);
    if (rc) return rc;
    if (se != cudaSuccess)
        return set_err(h, SNAC_GPU_ECUDA, -1, "cudaStreamSynchronize: %s", cudaGetErrorString(se));
    return 0;
}

// ======================================================================================
// Adjoint: gradients of a top-surface misfit with respect to the per-element
// cohesion, friction and viscosity scales, with checkpointing every K steps
// and recomputation of each segment before its reverse sweep.
// ======================================================================================
namespace {

struct Snap {
    double4* pos = nullptr;
    double4* vel = nullptr;
    double4* force = nullptr;
    double* stress = nullptr;
    double* eps_p = nullptr;
    DevScalars* sc = nullptr;
    double* vol = nullptr;  // Maxwell: the tet volumes and old volumes
    bool pending = false;
    long long time_step = 0;
};

int snap_alloc(snac_gpu* h, Snap& z) {
    const long long nn = h->mesh.nn, nq = h->mesh.ne * NT;
    int rc;
    if ((rc = dalloc(h, &z.pos, nn)) || (rc = dalloc(h, &z.vel, nn)) || (rc = dalloc(h, &z.force, nn)) ||
        (rc = dalloc(h, &z.stress, nq * 6)) || (rc = dalloc(h, &z.sc, 1)))
        return rc;
    // the hooks' own per-tet state: plastic strain (plastic, visco-plastic), volumes (Maxwell)
    if (h->eps_p && (rc = dalloc(h, &z.eps_p, nq))) return rc;
    if (h->vol && (rc = dalloc(h, &z.vol, nq * 2))) return rc;
    return 0;
}

void snap_free(Snap& z) {
    void* b[] = {z.pos, z.vel, z.force, z.stress, z.eps_p, z.sc, z.vol};
    for (void* p : b)
        if (p) cudaFree(p);
    z = Snap();
}

// one launch copying the arrays of a state (sizes in 64-bit words)
int snap_copy(snac_gpu* h, bool save, Snap& z) {
    static_assert(sizeof(DevScalars) % 8 == 0, "scalars are copied as 64-bit words");
    const long long nn = h->mesh.nn, nq = h->mesh.ne * NT;
    using U = unsigned long long;
    U* hp[7] = {(U*)h->pos[h->parity], (U*)h->vel, (U*)h->force, (U*)h->stress, (U*)h->eps_p, (U*)h->sc, (U*)h->vol};
    U* zp[7] = {(U*)z.pos, (U*)z.vel, (U*)z.force, (U*)z.stress, (U*)z.eps_p, (U*)z.sc, (U*)z.vol};
    const long long n[7] = {nn * 4, nn * 4, nn * 4, nq * 6, nq, (long long)(sizeof(DevScalars) / 8), nq * 2};
    CopyJob J;
    J.count = 0;
    for (int a = 0; a < 7; a++) {
        if (!hp[a] || !zp[a]) continue;  // a per-tet array this hook does not keep
        J.dst[J.count] = save ? zp[a] : hp[a];
        J.src[J.count] = save ? hp[a] : zp[a];
        J.n[J.count] = n[a];
        J.count++;
    }
    k_copy_many<<<148 * 8, 256, 0, h->stream>>>(J);
    h->launches++;
    int rc = launch_check_named(h, "k_copy_many");
    if (rc) return rc;
    if (save) {
        z.pending = h->pending;
        z.time_step = h->time_step;
    } else {
        h->pending = z.pending;
        h->time_step = z.time_step;
        h->hflux_ready = false;  // the heat-flux rows are not part of a snapshot
    }
    return 0;
}

int snap_save(snac_gpu* h, Snap& z) { return snap_copy(h, true, z); }
int snap_restore(snac_gpu* h, const Snap& z) { return snap_copy(h, false, const_cast<Snap&>(z)); }

AdjState adj_state(const Snap& z) { return AdjState{z.pos, z.vel, z.force, z.stress, z.eps_p, z.vol}; }

int adjoint_supported(snac_gpu* h) {
    if (!h->zero_done) return set_err(h, SNAC_GPU_ESTATE, -1, "adjoint: time step zero must come first");
    if (h->dp)
        return set_err(h, SNAC_GPU_ENOTSUP, -1, "adjoint: the Drucker-Prager return map is not differentiated");
    if (h->cfg.dt_type != SNAC_DT_CONSTANT)
        return set_err(h, SNAC_GPU_ENOTSUP, -1, "adjoint: dtType must be constant (dt may not depend on the state)");
    if (h->has_density || h->cfg.thermal_stress || h->cfg.winkler || h->cfg.traction || topo_on(h->cfg))
        return set_err(h, SNAC_GPU_ENOTSUP, -1,
                       "adjoint: density coupling, thermal stress, force-BC plugins and topography diffusion are not differentiated");
    if (h->temperature) {
        std::vector<DevMaterial> dm(MAX_PHASES);
        CK(cudaMemcpy(dm.data(), h->mats, MAX_PHASES * sizeof(DevMaterial), cudaMemcpyDeviceToHost));
        for (int p = 0; p < h->n_phases; p++)
            if (dm[p].thermal_conduct != 0.0)
                return set_err(h, SNAC_GPU_ENOTSUP, -1,
                               "adjoint: the temperature is held fixed; phase %d has thermal_conduct != 0", p);
    }
    return 0;
}

template <int P>
int adj_tet_launch_p(snac_gpu* h, const Fields& F, const AdjState& S, const AdjBufs& B, int rotate, int first_rev,
                     double dt) {
    const size_t smem = SNAC_ADJ_SMEM_REC ? (size_t)ELEM_WARPS * 32 * sizeof(ConsRec) : 0;
    if (smem > 48 * 1024) CK(cudaFuncSetAttribute(k_adj_tet<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_adj_tet<P><<<elem_blocks(h->mesh), ELEM_WARPS * 32, smem, h->stream>>>(h->mesh, F, h->cfg, S, B, rotate, first_rev,
                                                                              dt);
    return 0;
}

int adj_tet_launch(snac_gpu* h, const AdjState& S, const AdjBufs& B, int rotate, int first_rev, double dt) {
    const Fields F = fields(h);
    int rc;
    switch (h->constitutive) {
        case SNAC_RHEOLOGY_ELASTIC: rc = adj_tet_launch_p<SNAC_RHEOLOGY_ELASTIC>(h, F, S, B, rotate, first_rev, dt); break;
        case SNAC_RHEOLOGY_PLASTIC: rc = adj_tet_launch_p<SNAC_RHEOLOGY_PLASTIC>(h, F, S, B, rotate, first_rev, dt); break;
        case SNAC_RHEOLOGY_MAXWELL: rc = adj_tet_launch_p<SNAC_RHEOLOGY_MAXWELL>(h, F, S, B, rotate, first_rev, dt); break;
        default: rc = adj_tet_launch_p<SNAC_RHEOLOGY_VISCOPLASTIC>(h, F, S, B, rotate, first_rev, dt);
    }
    if (rc) return rc;
    h->launches++;
    return launch_check_named(h, "k_adj_tet");
}

int adj_nodes_launch(snac_gpu* h, const AdjState& cur, const AdjState& prev, const AdjBufs& B, int gather, int update,
                     double dt) {
    k_adj_nodes<<<(unsigned)((h->mesh.nn + 127) / 128), 128, 0, h->stream>>>(h->mesh, fields(h), cur, prev, B, gather,
                                                                           update, dt, h->cfg.demf);
    h->launches++;
    return launch_check_named(h, "k_adj_nodes");
}

int misfit(snac_gpu* h, const snac_adjoint_desc* a, const AdjBufs& B, double* terms_dev, double* loss) {
    const long long nt = (long long)h->mesh.nnx * h->mesh.nnz;
    double *tv = nullptr, *ty = nullptr;
    int rc;
    if ((rc = dalloc(h, &tv, nt)) || (rc = dalloc(h, &ty, nt))) {
        if (tv) cudaFree(tv);
        return rc;
    }
    cudaMemcpyAsync(tv, a->target_vy, nt * sizeof(double), cudaMemcpyHostToDevice, h->stream);
    cudaMemcpyAsync(ty, a->target_y, nt * sizeof(double), cudaMemcpyHostToDevice, h->stream);
    k_adj_loss<<<(unsigned)((h->mesh.nn + 127) / 128), 128, 0, h->stream>>>(h->mesh, h->pos[h->parity], h->vel, tv, ty,
                                                                          a->w_v, a->w_h, terms_dev, B);
    h->launches++;
    rc = launch_check_named(h, "k_adj_loss");
    std::vector<double> t(nt);
    cudaError_t e = cudaMemcpyAsync(t.data(), terms_dev, nt * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(tv);
    cudaFree(ty);
    if (rc) return rc;
    if (e != cudaSuccess) return set_err(h, SNAC_GPU_ECUDA, -1, "misfit: %s", cudaGetErrorString(e));
    double L = 0.0;
    for (long long i = 0; i < nt; i++) L += t[i];
    *loss = L;
    return 0;
}

struct AdjWork {
    AdjBufs B{};
    double* terms = nullptr;
    double* grads = nullptr;  // [3][ne]
    void release() {
        void* b[] = {B.xbar, B.vbar, B.fbar, B.cbuf, B.sbar, B.epbar, B.pbar, B.vobar, terms, grads};
        for (void* p : b)
            if (p) cudaFree(p);
        *this = AdjWork();
    }
};

int adj_work_alloc(snac_gpu* h, AdjWork& w) {
    const long long nn = h->mesh.nn, nq = h->mesh.ne * NT, nt = (long long)h->mesh.nnx * h->mesh.nnz;
    int rc;
    if ((rc = dalloc(h, &w.B.xbar, nn)) || (rc = dalloc(h, &w.B.vbar, nn)) || (rc = dalloc(h, &w.B.fbar, nn)) ||
        (rc = dalloc(h, &w.B.cbuf, h->mesh.ner * NT * 24)) || (rc = dalloc(h, &w.B.sbar, nq * 6)) || (rc = dalloc(h, &w.B.epbar, nq)) ||
        (rc = dalloc(h, &w.B.pbar, nq * 3)) || (rc = dalloc(h, &w.terms, nt)) || (rc = dalloc(h, &w.grads, 3 * h->mesh.ne)))
        return rc;
    if (h->constitutive == SNAC_RHEOLOGY_MAXWELL && (rc = dalloc(h, &w.B.vobar, nq))) return rc;
    return 0;
}

int adj_status(snac_gpu* h) {
    DevScalars sc;
    CK(cudaMemcpyAsync(&sc, h->sc, sizeof sc, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (sc.status == SNAC_GPU_ENOTSUP)
        return set_err(h, SNAC_GPU_ENOTSUP, sc.err_index,
                       "adjoint: element %lld left the softening table or has a friction angle <= 0", sc.err_index);
    return read_status(h);
}

}  // namespace

extern "C" {

int snac_gpu_misfit(snac_gpu* h, const snac_adjoint_desc* a, double* loss) {
    if (!h || !a || !loss || !a->target_vy || !a->target_y) return SNAC_GPU_EINVAL;
    AdjWork w;
    int rc = 0;
    const long long nn = h->mesh.nn, nt = (long long)h->mesh.nnx * h->mesh.nnz;
    if ((rc = dalloc(h, &w.B.xbar, nn)) || (rc = dalloc(h, &w.B.vbar, nn)) || (rc = dalloc(h, &w.B.fbar, nn)) ||
        (rc = dalloc(h, &w.terms, nt))) {
        w.release();
        return rc;
    }
    rc = misfit(h, a, w.B, w.terms, loss);
    w.release();
    return rc;
}

int snac_gpu_adjoint(snac_gpu* h, const snac_adjoint_desc* a, double* loss, double* grad_cohesion,
                     double* grad_friction, double* grad_viscosity, snac_adjoint_stats* stats) {
    snac_adjoint_grads g{};
    g.cohesion = grad_cohesion;
    g.friction = grad_friction;
    g.viscosity = grad_viscosity;
    return snac_gpu_adjoint_grads(h, a, loss, &g, stats);
}

int snac_gpu_adjoint_grads(snac_gpu* h, const snac_adjoint_desc* a, double* loss, const snac_adjoint_grads* gr,
                           snac_adjoint_stats* stats) {
    if (!h || !a || !loss || !gr || !a->target_vy || !a->target_y || a->nsteps < 1) return SNAC_GPU_EINVAL;
    int rc = adjoint_supported(h);
    if (rc) return rc;
    const int N = a->nsteps;
    int K = a->checkpoint_every > 0 ? a->checkpoint_every : (int)std::ceil(std::sqrt((double)N));
    if (K > N) K = N;
    const int ncp = (N + K - 1) / K;  // checkpoints at steps 0, K, 2K, ...
    const double dt = [&] {
        DevScalars sc;
        cudaMemcpy(&sc, h->sc, sizeof sc, cudaMemcpyDeviceToHost);
        return sc.dt;
    }();
    if ((rc = flush_pending(h))) return rc;

    std::vector<Snap> cp(ncp), seg(K + 1);
    Snap fin;
    AdjWork w;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    auto cleanup = [&]() {
        cudaStreamSynchronize(h->stream);
        for (auto& z : cp) snap_free(z);
        for (auto& z : seg) snap_free(z);
        snap_free(fin);
        w.release();
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
    };
#define ACK(x)              \
    do {                    \
        int rc_ = (x);      \
        if (rc_) {          \
            cleanup();      \
            return rc_;     \
        }                   \
    } while (0)
    for (auto& z : cp) ACK(snap_alloc(h, z));
    for (auto& z : seg) ACK(snap_alloc(h, z));
    ACK(snap_alloc(h, fin));
    ACK(adj_work_alloc(h, w));
    for (auto& e : ev)
        if (cudaEventCreate(&e) != cudaSuccess) ACK(set_err(h, SNAC_GPU_ECUDA, -1, "cudaEventCreate"));

    // forward sweep, keeping every K-th state
    cudaEventRecord(ev[0], h->stream);
    ACK(snap_save(h, cp[0]));
    for (int k = 1; k <= N; k++) {
        ACK(launch_step(h));
        if (k % K == 0 && k / K < ncp) ACK(snap_save(h, cp[k / K]));
    }
    ACK(snap_save(h, fin));
    cudaEventRecord(ev[1], h->stream);
    ACK(read_status(h));
    ACK(misfit(h, a, w.B, w.terms, loss));  // also seeds the node adjoints

    // reverse sweep, segment by segment from the last
    const long long nq = h->mesh.ne * NT;
    cudaMemsetAsync(w.B.sbar, 0, nq * 6 * sizeof(double), h->stream);
    cudaMemsetAsync(w.B.epbar, 0, nq * sizeof(double), h->stream);
    cudaMemsetAsync(w.B.pbar, 0, nq * 3 * sizeof(double), h->stream);
    if (w.B.vobar) cudaMemsetAsync(w.B.vobar, 0, nq * sizeof(double), h->stream);
    cudaEventRecord(ev[2], h->stream);
    for (int j = ncp - 1; j >= 0; j--) {
        const int a0 = j * K, b0 = std::min(a0 + K, N);
        ACK(snap_restore(h, cp[j]));
        std::swap(seg[0], cp[j]);  // the checkpoint is the segment's first state
        for (int k = a0 + 1; k <= b0; k++) {
            ACK(launch_step(h));
            ACK(snap_save(h, seg[k - a0]));
        }
        // reverse of the node update of step b0-1
        ACK(adj_nodes_launch(h, adj_state(seg[b0 - a0]), adj_state(seg[b0 - 1 - a0]), w.B, 0, 1, dt));
        for (int n = b0 - 1; n >= a0; n--) {
            ACK(adj_tet_launch(h, adj_state(seg[n - a0]), w.B, n >= 1, n == N - 1, dt));
            if (n > a0)
                ACK(adj_nodes_launch(h, adj_state(seg[n - a0]), adj_state(seg[n - 1 - a0]), w.B, 1, 1, dt));
            else
                ACK(adj_nodes_launch(h, adj_state(seg[0]), adj_state(seg[0]), w.B, 1, 0, dt));
        }
    }
    const long long ne = h->mesh.ne;
    k_adj_reduce<<<(unsigned)((ne + 127) / 128), 128, 0, h->stream>>>(ne, w.B.pbar, w.grads, w.grads + ne,
                                                                    w.grads + 2 * ne);
    h->launches++;
    ACK(launch_check_named(h, "k_adj_reduce"));
    cudaEventRecord(ev[3], h->stream);
    ACK(adj_status(h));
    if (gr->cohesion) cudaMemcpyAsync(gr->cohesion, w.grads, ne * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    if (gr->friction)
        cudaMemcpyAsync(gr->friction, w.grads + ne, ne * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    if (gr->viscosity)
        cudaMemcpyAsync(gr->viscosity, w.grads + 2 * ne, ne * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    // the adjoints the sweep left for the entry state (pass 0 wrote sbar and epbar,
    // the last node gather xbar and vbar)
    if (gr->coordinates) ACK(node_out(h, w.B.xbar, gr->coordinates, 0));
    if (gr->velocity) ACK(node_out(h, w.B.vbar, gr->velocity, 0));
    if (gr->stress) cudaMemcpyAsync(gr->stress, w.B.sbar, nq * 6 * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    if (gr->plastic_strain) {
        if (h->eps_p)
            cudaMemcpyAsync(gr->plastic_strain, w.B.epbar, nq * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
        else
            memset(gr->plastic_strain, 0, nq * sizeof(double));
    }
    // leave the model at the forward's final state
    ACK(snap_restore(h, fin));
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) ACK(set_err(h, SNAC_GPU_ECUDA, -1, "adjoint: sync"));
    if (stats) {
        float f = 0, r = 0;
        cudaEventElapsedTime(&f, ev[0], ev[1]);
        cudaEventElapsedTime(&r, ev[2], ev[3]);
        stats->ms_forward = f;
        stats->ms_reverse = r;
        stats->checkpoint_every = K;
        stats->checkpoints = ncp;
    }
    cleanup();
#undef ACK
    return 0;
}

}  // extern "C"

// ======================================================================================
// Dump and checkpoint files in the reference's format
// ======================================================================================
namespace {

const char* const kOutName[OutputState::NF] = {
    "strainRate", "stress", "hydroPressure", "phaseIndex", "coord", "vel", "force", "stressTensor", "plStrain",
    "viscosity", "temperature", "phaseIndexCP", "coordCP", "velCP", "stressTensorCP", "plStrainCP", "viscosityCP",
    "temperatureCP", "timeStep", "checkpointTimeStep", "sim"};

void output_join(OutputState* o) {
    if (o->writer.joinable()) o->writer.join();
}

// runs on the writer thread once the device records are in pinned memory
void output_write(OutputState* o) {
    if (cudaEventSynchronize(o->ready) != cudaSuccess) {
        o->err = SNAC_GPU_ECUDA;
        return;
    }
    for (const auto& p : o->pieces)
        if (o->f[p.file] && fwrite(o->pinned + p.off, 1, p.bytes, o->f[p.file]) != p.bytes) o->err = SNAC_GPU_EINVAL;
    DevScalars sc;
    memcpy(&sc, o->pinned + o->scal_off, sizeof sc);
    // Context.c:1286-1298 (rank 0 only): timeStep, currentTime, dt after Sync
    char line[128];
    snprintf(line, sizeof line, "%16u %16g %16g\n", (unsigned)sc.time_step, sc.current_time, sc.dt);
    if (o->dump && o->f[OutputState::T_STEP]) fputs(line, o->f[OutputState::T_STEP]);
    if (o->cp && o->f[OutputState::T_CP]) fputs(line, o->f[OutputState::T_CP]);
    for (FILE* f : o->f)
        if (f) fflush(f);
}

}  // namespace

extern "C" {

int snac_gpu_output_open(snac_gpu* h, const char* output_path, unsigned rank, unsigned dump_every,
                         unsigned checkpoint_every, unsigned max_time_steps) {
    if (!h || !output_path || dump_every == 0) return SNAC_GPU_EINVAL;
    if (h->out) return set_err(h, SNAC_GPU_ESTATE, -1, "output files are already open");
    OutputState* o = new (std::nothrow) OutputState();
    if (!o) return SNAC_GPU_ENOMEM;
    o->dir = output_path;
    o->rank = rank;
    o->dump_every = dump_every;
    o->checkpoint_every = checkpoint_every;
    o->max_steps = max_time_steps;
    const bool plastic = h->constitutive == SNAC_RHEOLOGY_PLASTIC || h->constitutive == SNAC_RHEOLOGY_VISCOPLASTIC;
    // viscosity records: SnacViscoPlastic's (viscoplastic/Output.c) and SnacMaxwell's (maxwell/Output.c)
    const bool visc = h->constitutive == SNAC_RHEOLOGY_VISCOPLASTIC || h->constitutive == SNAC_RHEOLOGY_MAXWELL;
    for (int i = 0; i < OutputState::NF; i++) {
        if ((i == OutputState::D_PL || i == OutputState::C_PL) && !plastic) continue;
        if ((i == OutputState::D_VI || i == OutputState::C_VI) && !visc) continue;
        if ((i == OutputState::D_TE || i == OutputState::C_TE) && !h->temperature) continue;
        if (i >= OutputState::T_STEP && rank != 0) continue;  // rank 0 only, Context.c:429-463
        std::string fn = o->dir + "/" + kOutName[i] + "." + std::to_string(rank);
        o->f[i] = fopen(fn.c_str(), "w+");
        if (!o->f[i]) {
            for (FILE* f : o->f)
                if (f) fclose(f);
            delete o;
            return set_err(h, SNAC_GPU_EINVAL, -1, "cannot open %s for writing", fn.c_str());
        }
    }
    if (o->f[OutputState::T_SIM]) {  // Context.c:431-446, one rank: the local counts are the global ones
        fprintf(o->f[OutputState::T_SIM],
                "%u %u %u %u %u %u %u %u %u\n(global element numbers)[3]=(proc numbers)[3]*(local element numbers)[3]\n",
                h->mesh.nx, h->mesh.ny, h->mesh.nz, 1u, 1u, 1u, h->mesh.nx, h->mesh.ny, h->mesh.nz);
        fflush(o->f[OutputState::T_SIM]);
    }
    // staging: the largest write is a dump plus a checkpoint at the same step
    const long long ne = h->mesh.ne, nn = h->mesh.nn;
    const size_t need = (size_t)(ne * (4 + 1 + 6 + 1 + 1) + nn * (3 * 3 + 1) + ne * (1 + 60 + 10 + 10) + nn * (3 * 2 + 1)) * 4 +
                        sizeof(DevScalars) + 256 * 24;
    cudaError_t e = cudaMalloc((void**)&o->dstage, need);
    if (e == cudaSuccess) h->alloc_bytes += (long long)need;
    if (e == cudaSuccess) e = cudaMallocHost((void**)&o->pinned, need);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&o->ready, cudaEventDisableTiming);
    if (e == cudaSuccess && !h->escal) {
        e = cudaMalloc((void**)&h->escal, ne * 4 * sizeof(double));
        if (e == cudaSuccess) h->alloc_bytes += ne * 4 * (long long)sizeof(double);
        if (e == cudaSuccess) e = cudaMemsetAsync(h->escal, 0, ne * 4 * sizeof(double), h->stream);
    }
    o->cap = need;
    h->out = o;
    if (e != cudaSuccess) {
        snac_gpu_output_close(h);
        return set_err(h, SNAC_GPU_ENOMEM, -1, "output staging: %s", cudaGetErrorString(e));
    }
    // the graphs hold the field pointers: re-capture them with the element-scalar buffer
    for (auto& gr : h->graph)
        for (auto& gf : gr)
            for (auto& g : gf)
                if (g) {
                    cudaGraphExecDestroy(g);
                    g = nullptr;
                }
    return 0;
}

int snac_gpu_write_output(snac_gpu* h) {
    if (!h) return SNAC_GPU_EINVAL;
    OutputState* o = h->out;
    if (!o) return set_err(h, SNAC_GPU_ESTATE, -1, "snac_gpu_output_open must come first");
    const long long ts = h->time_step;
    const bool dump = time_to_dump(o, ts), cp = time_to_checkpoint(o, ts);
    if (!dump && !cp) return 0;
    output_join(o);  // the previous write has left the pinned buffer
    if (o->err) return set_err(h, o->err, -1, "writing the output files failed");
    int rc = flush_pending(h);  // the files hold the end-of-step state
    if (rc) return rc;
    o->dump = dump;
    o->cp = cp;
    o->pieces.clear();
    size_t off = 0;
    auto take = [&](int file, size_t bytes) -> char* {
        if (!o->f[file]) return nullptr;
        char* p = o->dstage + off;
        o->pieces.push_back({file, off, bytes});
        off = (off + bytes + 255) & ~(size_t)255;
        return p;
    };
    const long long ne = h->mesh.ne, nn = h->mesh.nn;
    using S = OutputState;
    float *co = nullptr, *ve = nullptr, *fo = nullptr, *te = nullptr, *cco = nullptr, *cve = nullptr, *cte = nullptr;
    ElemOut E{};
    E.maxwell = h->constitutive == SNAC_RHEOLOGY_MAXWELL;
    if (dump) {
        E.strain_rate = (float*)take(S::D_SR, ne * 4);
        E.stress = (float*)take(S::D_ST, ne * 4);
        E.hydro_pressure = (float*)take(S::D_HP, ne * 4);
        E.tensor = (float*)take(S::D_TEN, ne * 24);
        co = (float*)take(S::D_CO, nn * 12);
        ve = (float*)take(S::D_VE, nn * 12);
        fo = (float*)take(S::D_FO, nn * 12);
        E.phase = (int*)take(S::D_PH, ne * 4);
        E.aps = (float*)take(S::D_PL, ne * 4);
        E.log_visc = (float*)take(S::D_VI, ne * 4);
        te = (float*)take(S::D_TE, nn * 4);
    }
    if (cp) {
        E.tensor_cp = (float*)take(S::C_TEN, ne * 240);
        cco = (float*)take(S::C_CO, nn * 12);
        cve = (float*)take(S::C_VE, nn * 12);
        E.phase_cp = (int*)take(S::C_PH, ne * 4);
        E.eps_cp = (float*)take(S::C_PL, ne * 40);
        E.log_visc_cp = (float*)take(S::C_VI, ne * (h->constitutive == SNAC_RHEOLOGY_MAXWELL ? 4 : 40));
        cte = (float*)take(S::C_TE, nn * 4);
    }
    o->scal_off = off;
    off += sizeof(DevScalars);
    if (off > o->cap) return set_err(h, SNAC_GPU_EINVAL, -1, "output staging too small");
    const Fields F = fields(h);
    const unsigned nb = (unsigned)((nn + 255) / 256), eb = (unsigned)((ne + 127) / 128);
    if (co || ve || fo || te) {
        k_out_nodes<<<nb, 256, 0, h->stream>>>(F.pos, F.vel, F.force, nn, co, ve, fo, te);
        h->launches++;
        if ((rc = launch_check_named(h, "k_out_nodes"))) return rc;
    }
    if (cco || cve || cte) {
        k_out_nodes<<<nb, 256, 0, h->stream>>>(F.pos, F.vel, F.force, nn, cco, cve, nullptr, cte);
        h->launches++;
        if ((rc = launch_check_named(h, "k_out_nodes"))) return rc;
    }
    k_out_elements<<<eb, 128, 0, h->stream>>>(h->mesh, F, E);
    h->launches++;
    if ((rc = launch_check_named(h, "k_out_elements"))) return rc;
    CK(cudaMemcpyAsync(o->dstage + o->scal_off, h->sc, sizeof(DevScalars), cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaMemcpyAsync(o->pinned, o->dstage, off, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaEventRecord(o->ready, h->stream));
    o->writer = std::thread(output_write, o);
    return 0;
}

int snac_gpu_output_close(snac_gpu* h) {
    if (!h || !h->out) return h ? 0 : SNAC_GPU_EINVAL;
    OutputState* o = h->out;
    output_join(o);
    const int err = o->err;
    for (FILE* f : o->f)
        if (f) fclose(f);
    if (o->dstage) cudaFree(o->dstage);
    if (o->pinned) cudaFreeHost(o->pinned);
    if (o->ready) cudaEventDestroy(o->ready);
    delete o;
    h->out = nullptr;
    return err ? set_err(h, err, -1, "writing the output files failed") : 0;
}

}  // extern "C"
