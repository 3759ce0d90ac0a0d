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
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "snac_gpu.h"
#include "snac_kernels.cuh"

using namespace snac;

struct snac_gpu {
    Mesh mesh{};
    Config cfg{};
    int constitutive = 0;
    int temperature = 0;
    int has_density = 0;
    int n_phases = 0;
    double wave_speed = 0.0;
    cudaStream_t stream = nullptr;
    // device buffers
    double4* pos[2] = {nullptr, nullptr};
    double4* vel = nullptr;
    double4* force = nullptr;
    double* stress = nullptr;
    double* eps_p = nullptr;
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
    // host mirror of the step bookkeeping
    int parity = 0;
    long long time_step = 0;
    bool zero_done = false;
    cudaGraphExec_t graph[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};  // [fused][parity]
    bool pending = false;  // the element update of the last step is deferred into the next kernel
    // kernel-by-kernel timing (snac_gpu_profile_step)
    snac_kernel_time* prof = nullptr;
    int prof_n = 0, prof_max = 0;
    cudaEvent_t prof_ev[64];
    long long launches = 0;
    int steps_kernels[2] = {0, 0};
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
DevMaterial to_dev(const snac_material& s, bool fric_scaled) {
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
    return d;
}

Fields fields(snac_gpu* h) {
    Fields F;
    F.pos = h->pos[h->parity];
    F.pos_next = h->pos[h->parity ^ 1];
    F.vel = h->vel;
    F.force = h->force;
    F.stress = h->stress;
    F.eps_p = h->eps_p;
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
    F.coh_scale = h->coh_scale;
    F.fric_scale = h->fric_scale;
    F.visc_scale = h->visc_scale;
    F.sc = h->sc;
    return F;
}

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

template <int P>
void launch_stress(snac_gpu* h, const Fields& F, const Config& c) {
    k_calc_stresses<P><<<elem_blocks(h->mesh), ELEM_WARPS * 32, 0, h->stream>>>(h->mesh, F, c);
}
template <int P>
void launch_update(snac_gpu* h, const Fields& F, const Config& c, int pending) {
    k_update_elements<P><<<elem_blocks(h->mesh), ELEM_WARPS * 32, 0, h->stream>>>(h->mesh, F, c, pending);
}
template <int P>
void launch_fused(snac_gpu* h, const Fields& F, const Config& c) {
    k_fused_step<P><<<elem_blocks(h->mesh), ELEM_WARPS * 32, 0, h->stream>>>(h->mesh, F, c);
}
template <int P>
void launch_fused_heat(snac_gpu* h, const Fields& F, const Config& c) {
    k_fused_heat<P><<<elem_blocks(h->mesh), ELEM_WARPS * 32, 0, h->stream>>>(h->mesh, F, c);
}

int op_energy_elements(snac_gpu* h) {
    if (!h->temperature) return 0;
    k_heat_flux<<<elem_blocks(h->mesh), ELEM_WARPS * 32, 0, h->stream>>>(h->mesh, fields(h), h->cfg);
    h->launches++;
    return launch_check_named(h, "k_heat_flux");
}

int op_energy_nodes(snac_gpu* h) {
    if (!h->temperature) return 0;
    k_heat_nodes<<<node_blocks(h->mesh), 128, 0, h->stream>>>(h->mesh, fields(h), h->cfg);
    h->launches++;
    return launch_check_named(h, "k_heat_nodes");
}

int op_calc_stresses(snac_gpu* h) {
    Fields F = fields(h);
    switch (h->constitutive) {
        case SNAC_RHEOLOGY_ELASTIC: launch_stress<SNAC_RHEOLOGY_ELASTIC>(h, F, h->cfg); break;
        case SNAC_RHEOLOGY_PLASTIC: launch_stress<SNAC_RHEOLOGY_PLASTIC>(h, F, h->cfg); break;
        case SNAC_RHEOLOGY_VISCOPLASTIC: launch_stress<SNAC_RHEOLOGY_VISCOPLASTIC>(h, F, h->cfg); break;
        case SNAC_RHEOLOGY_MAXWELL: launch_stress<SNAC_RHEOLOGY_MAXWELL>(h, F, h->cfg); break;
    }
    h->launches++;
    return launch_check_named(h, "k_calc_stresses");
}

int op_loop_nodes(snac_gpu* h) {
    Fields F = fields(h);
    unsigned nb = node_blocks(h->mesh);
    switch (h->cfg.dt_type) {
        case SNAC_DT_CONSTANT: k_loop_nodes<SNAC_DT_CONSTANT><<<nb, 128, 0, h->stream>>>(h->mesh, F, h->cfg); break;
        case SNAC_DT_DYNAMIC: k_loop_nodes<SNAC_DT_DYNAMIC><<<nb, 128, 0, h->stream>>>(h->mesh, F, h->cfg); break;
        default: k_loop_nodes<SNAC_DT_WAVE><<<nb, 128, 0, h->stream>>>(h->mesh, F, h->cfg); break;
    }
    h->launches++;
    h->parity ^= 1;  // the new coordinates are current from here on
    return launch_check_named(h, "k_loop_nodes");
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

// the end of the previous step fused with the start of this one
int op_fused(snac_gpu* h) {
    Fields F = fields(h);
    Config c = h->cfg;
    c.time_step_zero = 0;
    if (h->temperature) {
        switch (h->constitutive) {
            case SNAC_RHEOLOGY_MAXWELL: launch_fused_heat<SNAC_RHEOLOGY_MAXWELL>(h, F, c); break;
            default: launch_fused_heat<SNAC_RHEOLOGY_ELASTIC>(h, F, c); break;
        }
    } else {
        switch (h->constitutive) {
            case SNAC_RHEOLOGY_ELASTIC: launch_fused<SNAC_RHEOLOGY_ELASTIC>(h, F, c); break;
            case SNAC_RHEOLOGY_PLASTIC: launch_fused<SNAC_RHEOLOGY_PLASTIC>(h, F, c); break;
            case SNAC_RHEOLOGY_VISCOPLASTIC: launch_fused<SNAC_RHEOLOGY_VISCOPLASTIC>(h, F, c); break;
            case SNAC_RHEOLOGY_MAXWELL: launch_fused<SNAC_RHEOLOGY_MAXWELL>(h, F, c); break;
        }
    }
    h->launches++;
    h->time_step++;
    return launch_check_named(h, h->temperature ? "k_fused_heat" : "k_fused_step");
}

int op_min_length_scale(snac_gpu* h) {
    k_min_length_scale<<<(unsigned)((h->mesh.ne + 127) / 128), 128, 0, h->stream>>>(h->mesh, fields(h));
    h->launches++;
    return launch_check_named(h, "k_min_length_scale");
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
int record_step(snac_gpu* h, bool fused) {
    int rc;
    if (fused) {
        if ((rc = op_fused(h))) return rc;
    } else {
        if ((rc = op_begin(h))) return rc;
        if ((rc = op_energy_elements(h))) return rc;
    }
    if ((rc = op_energy_nodes(h))) return rc;
    if (fused && !h->temperature) {
        // stress already updated by the fused kernel
    } else if ((rc = op_calc_stresses(h))) {
        return rc;
    }
    if ((rc = op_loop_nodes(h))) return rc;
    if ((rc = op_min_length_scale(h))) return rc;
    return op_sync(h);
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

// hydroStaticIC/VariableConditions.c:43-152 on one rank: lithostatic
// pressure integrated down each element column; densities are the phase
// densities (tet densities are still zero at this point of the reference's IC).
void hydrostatic_ic(const snac_gpu_desc* d, const std::vector<double>& coord, std::vector<double>& stress) {
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
            }
        }
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

int snac_gpu_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
    return n;
}

int snac_gpu_create(const snac_gpu_desc* d, snac_gpu** out) {
    if (!out) return SNAC_GPU_EINVAL;
    *out = nullptr;
    if (!d || d->abi_version != SNAC_GPU_ABI_VERSION) return SNAC_GPU_EINVAL;
    if (d->nx < 1 || d->ny < 1 || d->nz < 1 || d->n_materials < 1 || !d->materials) return SNAC_GPU_EINVAL;
    if (d->n_materials > MAX_PHASES) return SNAC_GPU_EINVAL;
    if (d->constitutive != SNAC_RHEOLOGY_ELASTIC && d->constitutive != SNAC_RHEOLOGY_PLASTIC &&
        d->constitutive != SNAC_RHEOLOGY_VISCOPLASTIC && d->constitutive != SNAC_RHEOLOGY_MAXWELL)
        return SNAC_GPU_EINVAL;
    if ((d->constitutive == SNAC_RHEOLOGY_VISCOPLASTIC || d->constitutive == SNAC_RHEOLOGY_MAXWELL) && !d->temperature)
        return SNAC_GPU_EINVAL;  // both hooks read the temperature plugin's node extension
    if (d->dt_type < SNAC_DT_CONSTANT || d->dt_type > SNAC_DT_WAVE) return SNAC_GPU_EINVAL;
    bool per_elem = d->element_cohesion_scale || d->element_friction_scale || d->element_visc_scale;
    if (per_elem && d->constitutive == SNAC_RHEOLOGY_MAXWELL) return SNAC_GPU_ENOTSUP;
    for (int p = 0; p < d->n_materials; p++) {
        if (d->materials[p].nsegments < 0 || d->materials[p].nsegments > SNAC_MAX_SEGMENTS) return SNAC_GPU_EINVAL;
        if ((d->constitutive == SNAC_RHEOLOGY_PLASTIC || d->constitutive == SNAC_RHEOLOGY_VISCOPLASTIC) &&
            !d->materials[p].yield_mohr_coulomb)
            return SNAC_GPU_ENOTSUP;  // the Drucker-Prager branch is not built
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
    h->constitutive = d->constitutive;
    h->temperature = d->temperature;
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
    CK(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));

    const long long ne = m.ne, nn = m.nn, nq = ne * NT;
    int rc = 0;
    if ((rc = dalloc(h, &h->pos[0], nn)) || (rc = dalloc(h, &h->pos[1], nn)) || (rc = dalloc(h, &h->vel, nn)) ||
        (rc = dalloc(h, &h->force, nn)) || (rc = dalloc(h, &h->stress, nq * 6)) || (rc = dalloc(h, &h->bc, nn)) ||
        (rc = dalloc(h, &h->sc, 1)) || (rc = dalloc(h, &h->mats, MAX_PHASES)) ||
        (rc = dalloc(h, &h->fterm, nq * 12)) || (rc = dalloc(h, &h->fgrav, nq)) ||
        (rc = dalloc(h, &h->fmass, d->dt_type == SNAC_DT_CONSTANT ? nq * 4 : nq)))
        return rc;
    if (d->constitutive == SNAC_RHEOLOGY_PLASTIC || d->constitutive == SNAC_RHEOLOGY_VISCOPLASTIC)
        if ((rc = dalloc(h, &h->eps_p, nq))) return rc;
    if (d->constitutive == SNAC_RHEOLOGY_VISCOPLASTIC || d->constitutive == SNAC_RHEOLOGY_MAXWELL)
        if ((rc = dalloc(h, &h->visc, nq))) return rc;
    if (d->constitutive == SNAC_RHEOLOGY_MAXWELL)
        if ((rc = dalloc(h, &h->vol, nq * 2))) return rc;
    if (h->has_density)
        if ((rc = dalloc(h, &h->density, nq))) return rc;
    if (d->temperature) {
        if ((rc = dalloc(h, &h->hflux, nq * HF_STRIDE))) return rc;
        if (h->has_density && (rc = dalloc(h, &h->tpre, nn))) return rc;
    }

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
        for (int b = 0; b < d->n_velocity_bcs; b++) {  // last VC wins, CompositeVC.c:599-611
            const snac_wall_bc& w = d->velocity_bcs[b];
            if (!wall_has(w.wall, i, j, k, m.nnx, m.nny, m.nnz)) continue;
            for (int q = 0; q < 3; q++)
                if (w.mask & (1 << q)) idx[q] = (unsigned char)b;
        }
        for (int b = 0; b < d->n_temperature_bcs; b++) {
            const snac_wall_bc& w = d->temperature_bcs[b];
            if ((w.mask & 1) && wall_has(w.wall, i, j, k, m.nnx, m.nny, m.nnz)) idx[3] = (unsigned char)b;
        }
        bc[n] = make_uchar4(idx[0], idx[1], idx[2], idx[3]);
        // temperature0 = temperature before the BCs are applied
        // (_SnacTemperature_InitialConditions, temperature/VariableConditions.c:240-256)
        temp0[n] = temp[n];
        // VariableCondition_Apply(velocityBCs), Context.c:773
        for (int q = 0; q < 3; q++)
            if (idx[q] != 255) vel[n * 3 + q] = d->velocity_bcs[idx[q]].value[q];
        if (d->temperature && idx[3] != 255) temp[n] = d->temperature_bcs[idx[3]].value[0];
    }
    if (d->init_stress) std::copy(d->init_stress, d->init_stress + nq * 6, stress.begin());
    if (d->hydrostatic_ic) hydrostatic_ic(d, coord, stress);

    std::vector<double4> pos4(nn), vel4(nn);
    for (long long n = 0; n < nn; n++) {
        pos4[n] = make_double4(coord[n * 3], coord[n * 3 + 1], coord[n * 3 + 2], temp[n]);
        vel4[n] = make_double4(vel[n * 3], vel[n * 3 + 1], vel[n * 3 + 2], temp0[n]);
    }
    std::vector<double> vbc(std::max(1, d->n_velocity_bcs) * 3, 0.0), tbc(std::max(1, d->n_temperature_bcs), 0.0);
    for (int b = 0; b < d->n_velocity_bcs; b++)
        for (int q = 0; q < 3; q++) vbc[b * 3 + q] = d->velocity_bcs[b].value[q];
    for (int b = 0; b < d->n_temperature_bcs; b++) tbc[b] = d->temperature_bcs[b].value[0];
    if ((rc = dalloc(h, &h->vbc_val, vbc.size())) || (rc = dalloc(h, &h->tbc_val, tbc.size()))) return rc;

    std::vector<DevMaterial> dm(MAX_PHASES);
    for (int p = 0; p < d->n_materials; p++) dm[p] = to_dev(d->materials[p], d->element_friction_scale != nullptr);
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
    CK(cudaMemcpyAsync(h->sc, &sc, sizeof sc, cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return 0;
}

void snac_gpu_destroy(snac_gpu* h) {
    if (!h) return;
    if (h->stream) cudaStreamSynchronize(h->stream);
    for (auto& gf : h->graph)
        for (auto& g : gf)
            if (g) cudaGraphExecDestroy(g);
    void* bufs[] = {h->pos[0], h->pos[1], h->vel, h->force, h->stress, h->eps_p, h->visc, h->density, h->vol,
                    h->hflux, h->tpre, h->fterm, h->fgrav, h->fmass, h->bc, h->vbc_val, h->tbc_val, h->mat, h->mats, h->coh_scale, h->fric_scale,
                    h->visc_scale, h->sc};
    for (void* b : bufs)
        if (b) cudaFree(b);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

int snac_gpu_time_step_zero(snac_gpu* h) {
    if (!h) return SNAC_GPU_EINVAL;
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
        int p = h->parity, f = h->pending ? 1 : 0;
        if (!h->graph[f][p]) {
            cudaGraph_t g;
            long long l0 = h->launches, ts0 = h->time_step;
            CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
            int rc = record_step(h, f == 1);
            cudaError_t e = cudaStreamEndCapture(h->stream, &g);
            if (rc) return rc;
            if (e != cudaSuccess) return set_err(h, SNAC_GPU_ECUDA, -1, "graph capture: %s", cudaGetErrorString(e));
            CK(cudaGraphInstantiate(&h->graph[f][p], g, 0));
            cudaGraphDestroy(g);
            h->steps_kernels[f] = (int)(h->launches - l0);
            h->launches = l0;  // counted again below, when the graph actually runs
            h->time_step = ts0;
            h->parity = p;
        }
        CK(cudaGraphLaunch(h->graph[f][p], h->stream));
        h->launches += h->steps_kernels[f];
        h->time_step++;
        h->parity ^= 1;
        h->pending = true;
    }
    return read_status(h);
}

int snac_gpu_begin_step(snac_gpu* h) {
    if (!h) return SNAC_GPU_EINVAL;
    if (!h->zero_done) return set_err(h, SNAC_GPU_ESTATE, -1, "snac_gpu_time_step_zero must come first");
    int rc = flush_pending(h);
    return rc ? rc : op_begin(h);
}
int snac_gpu_loop_elements_energy(snac_gpu* h) {
    if (!h) return SNAC_GPU_EINVAL;
    int rc = flush_pending(h);
    return rc ? rc : op_energy_elements(h);
}
int snac_gpu_loop_nodes_energy(snac_gpu* h) {
    if (!h) return SNAC_GPU_EINVAL;
    int rc = flush_pending(h);
    return rc ? rc : op_energy_nodes(h);
}
int snac_gpu_calc_stresses(snac_gpu* h) {
    if (!h) return SNAC_GPU_EINVAL;
    int rc = flush_pending(h);
    if (!rc) rc = op_calc_stresses(h);
    return rc ? rc : read_status(h);
}
int snac_gpu_loop_nodes_momentum(snac_gpu* h) {
    if (!h) return SNAC_GPU_EINVAL;
    int rc = flush_pending(h);
    if (!rc) rc = op_loop_nodes(h);
    return rc ? rc : read_status(h);
}
int snac_gpu_loop_elements_momentum(snac_gpu* h) {
    if (!h) return SNAC_GPU_EINVAL;
    int rc = flush_pending(h);
    if (!rc) rc = op_update_elements(h, h->time_step == 0);
    return rc ? rc : read_status(h);
}
int snac_gpu_sync(snac_gpu* h) {
    if (!h) return SNAC_GPU_EINVAL;
    int rc = flush_pending(h);
    if (!rc) rc = op_sync_full(h);
    return rc ? rc : read_status(h);
}

int snac_gpu_upload(snac_gpu* h, const snac_state_view* v) {
    if (!h || !v) return SNAC_GPU_EINVAL;
    if (int rc = flush_pending(h)) return rc;
    const long long nn = h->mesh.nn, nq = h->mesh.ne * NT;
    if (v->coord || v->velocity || v->temperature) {
        std::vector<double4> p(nn), w(nn);
        CK(cudaMemcpy(p.data(), h->pos[h->parity], nn * sizeof(double4), cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(w.data(), h->vel, nn * sizeof(double4), cudaMemcpyDeviceToHost));
        for (long long n = 0; n < nn; n++) {
            if (v->coord) p[n] = make_double4(v->coord[n * 3], v->coord[n * 3 + 1], v->coord[n * 3 + 2], p[n].w);
            if (v->velocity) w[n] = make_double4(v->velocity[n * 3], v->velocity[n * 3 + 1], v->velocity[n * 3 + 2], w[n].w);
            if (v->temperature) p[n].w = v->temperature[n];
        }
        CK(cudaMemcpy(h->pos[h->parity], p.data(), nn * sizeof(double4), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(h->vel, w.data(), nn * sizeof(double4), cudaMemcpyHostToDevice));
    }
    if (v->stress) CK(cudaMemcpy(h->stress, v->stress, nq * 6 * sizeof(double), cudaMemcpyHostToDevice));
    if (v->plastic_strain && h->eps_p) CK(cudaMemcpy(h->eps_p, v->plastic_strain, nq * sizeof(double), cudaMemcpyHostToDevice));
    if (v->viscosity && h->visc) CK(cudaMemcpy(h->visc, v->viscosity, nq * sizeof(double), cudaMemcpyHostToDevice));
    return 0;
}

int snac_gpu_download(snac_gpu* h, const snac_state_view* v) {
    if (!h || !v) return SNAC_GPU_EINVAL;
    if (int rc = flush_pending(h)) return rc;
    CK(cudaStreamSynchronize(h->stream));
    const long long nn = h->mesh.nn, nq = h->mesh.ne * NT;
    if (v->coord || v->velocity || v->temperature || v->force || v->inertial_mass) {
        std::vector<double4> p(nn), w(nn), f(nn);
        CK(cudaMemcpy(p.data(), h->pos[h->parity], nn * sizeof(double4), cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(w.data(), h->vel, nn * sizeof(double4), cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(f.data(), h->force, nn * sizeof(double4), cudaMemcpyDeviceToHost));
        for (long long n = 0; n < nn; n++) {
            if (v->coord) {
                v->coord[n * 3] = p[n].x;
                v->coord[n * 3 + 1] = p[n].y;
                v->coord[n * 3 + 2] = p[n].z;
            }
            if (v->velocity) {
                v->velocity[n * 3] = w[n].x;
                v->velocity[n * 3 + 1] = w[n].y;
                v->velocity[n * 3 + 2] = w[n].z;
            }
            if (v->temperature) v->temperature[n] = p[n].w;
            if (v->force) {
                v->force[n * 3] = f[n].x;
                v->force[n * 3 + 1] = f[n].y;
                v->force[n * 3 + 2] = f[n].z;
            }
            if (v->inertial_mass) v->inertial_mass[n] = f[n].w;
        }
    }
    if (v->stress) CK(cudaMemcpy(v->stress, h->stress, nq * 6 * sizeof(double), cudaMemcpyDeviceToHost));
    if (v->plastic_strain) {
        if (h->eps_p)
            CK(cudaMemcpy(v->plastic_strain, h->eps_p, nq * sizeof(double), cudaMemcpyDeviceToHost));
        else
            memset(v->plastic_strain, 0, nq * sizeof(double));
    }
    if (v->viscosity) {
        if (h->visc)
            CK(cudaMemcpy(v->viscosity, h->visc, nq * sizeof(double), cudaMemcpyDeviceToHost));
        else
            memset(v->viscosity, 0, nq * sizeof(double));
    }
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
