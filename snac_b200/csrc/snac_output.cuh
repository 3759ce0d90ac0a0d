// snac_output.cuh — packing kernels of the dump and checkpoint files.
//
// The reference writes raw float32 (int32 for phase indices) records, one
// file per field and rank, appended at every dump / checkpoint step
// (Snac/libSnac/src/Context.c:1311-1531, StGermain's
// VariableDumpStream.c:137-190 for the node and element variables, the
// plugins' Output.c for plastic strain, viscosity and temperature).  These
// kernels produce those records on the device from the current state; the
// host copies them to pinned memory and appends them to the files.
#pragma once

#include "snac_kernels.cuh"

namespace snac {

// node records: coord / vel / force (3 floats per node), temperature (1)
__global__ void k_out_nodes(const double4* __restrict__ pos, const double4* __restrict__ vel,
                            const double4* __restrict__ force, long long nn, float* coord, float* velo, float* frc,
                            float* temp) {
    long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nn) return;
    const double4 p = pos[n];
    if (coord) {
        coord[n * 3 + 0] = (float)p.x;
        coord[n * 3 + 1] = (float)p.y;
        coord[n * 3 + 2] = (float)p.z;
    }
    if (velo) {
        const double4 w = vel[n];
        velo[n * 3 + 0] = (float)w.x;
        velo[n * 3 + 1] = (float)w.y;
        velo[n * 3 + 2] = (float)w.z;
    }
    if (frc) {
        const double4 f = force[n];
        frc[n * 3 + 0] = (float)f.x;
        frc[n * 3 + 1] = (float)f.y;
        frc[n * 3 + 2] = (float)f.z;
    }
    if (temp) temp[n] = (float)p.w;
}

struct ElemOut {
    // dump
    float *strain_rate, *stress, *hydro_pressure, *tensor, *aps, *log_visc;
    int* phase;
    // checkpoint
    float *tensor_cp, *eps_cp, *log_visc_cp;
    int* phase_cp;
    int maxwell;  // SnacMaxwell's viscosity records (maxwell/Output.c) instead of SnacViscoPlastic's
};

// element records: one thread per element
__global__ void k_out_elements(Mesh m, Fields F, ElemOut O) {
    long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m.ne) return;
    const int ph = phase_of(F, e);
    if (O.phase) O.phase[e] = ph;
    if (O.phase_cp) O.phase_cp[e] = ph;
    if (F.escal) {
        if (O.strain_rate) O.strain_rate[e] = (float)F.escal[e * 4 + 0];
        if (O.stress) O.stress[e] = (float)F.escal[e * 4 + 1];
        if (O.hydro_pressure) O.hydro_pressure[e] = (float)F.escal[e * 4 + 2];
        if (O.aps) O.aps[e] = (float)F.escal[e * 4 + 3];
    }
    const double* S = F.stress + e * NT * 6;
    if (O.tensor) {
        // Context.c:1469-1490: volume-weighted mean of the tet stresses, accumulated in float
        int i, j, k;
        elem_ijk(m, e, i, j, k);
        V3 corner[8];
#pragma unroll
        for (int cc = 0; cc < 8; cc++) {
            double4 p = F.pos[corner_node(m, i, j, k, cc)];
            corner[cc] = {p.x, p.y, p.z};
        }
        double V[NT];
#pragma unroll
        for (int t = 0; t < NT; t++)
            V[t] = tet_volume(corner[tet_node(t, 0)], corner[tet_node(t, 1)], corner[tet_node(t, 2)],
                              corner[tet_node(t, 3)]);
        float totalVolume = 0.0;
        for (int t = 0; t < NT; t++) totalVolume += V[t];
        float sv[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        for (int t = 0; t < NT; t++)
            for (int a = 0; a < 6; a++) sv[a] += S[t * 6 + a] * V[t] / totalVolume;
        for (int a = 0; a < 6; a++) O.tensor[e * 6 + a] = sv[a];
    }
    if (O.tensor_cp)
        for (int t = 0; t < NT; t++)
            for (int a = 0; a < 6; a++) O.tensor_cp[(e * NT + t) * 6 + a] = (float)S[t * 6 + a];
    if (O.eps_cp && F.eps_p)
        for (int t = 0; t < NT; t++) O.eps_cp[e * NT + t] = (float)F.eps_p[e * NT + t];
    if (O.maxwell && F.visc && (O.log_visc || O.log_visc_cp)) {
        // maxwell/Output.c:57-118: the tet mean accumulated in a float, its
        // log10 when positive; dump and checkpoint both write this one value
        float viscosity = 0.0f;
        for (int t = 0; t < NT; t++) viscosity += F.visc[e * NT + t] / NT;
        if (viscosity > 0.0) viscosity = (float)log10((double)viscosity);  // C: the float promotes to double
        if (O.log_visc) O.log_visc[e] = viscosity;
        if (O.log_visc_cp) O.log_visc_cp[e] = viscosity;
        return;
    }
    if (O.log_visc && F.visc) {
        // viscoplastic/Output.c: log10 of the mean tet viscosity
        double viscosity = 0.0f;
        for (int t = 0; t < NT; t++) viscosity += F.visc[e * NT + t] / NT;
        O.log_visc[e] = (float)log10(viscosity);
    }
    if (O.log_visc_cp && F.visc)
        for (int t = 0; t < NT; t++) O.log_visc_cp[e * NT + t] = (float)log10(F.visc[e * NT + t]);
}

}  // namespace snac
