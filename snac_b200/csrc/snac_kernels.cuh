// snac_kernels.cuh — the kernels of one SNAC step (reference rounding).
//
// Per step, in _Snac_Context_Solve order (Snac/libSnac/src/Context.c:1063-1099):
//   k_heat_flux      Snac_EP_LoopElementsEnergy  temperature/HeatFlux.c:47-200 + HeatFluxBC
//   k_heat_nodes     Snac_EP_LoopNodesEnergy     temperature/Heat.c:47-140
//   k_calc_stresses  Snac_EP_CalcStresses        StrainRate.c + Stress.c + the constitutive hook
//   k_loop_nodes     Snac_EP_LoopNodesMomentum   Force.c + UpdateNode.c
//   k_update_elements Snac_EP_LoopElementsMomentum UpdateElement.c
//   k_sync           AbstractContext_EP_Sync     Context.c:1208-1268
// In a steady step the element update of step n runs fused with the stress
// update of step n+1 (k_fused_step; with temperature k_heat_flux, k_heat_nodes,
// then k_fused_stress, since neither energy hook reads the stress), and the
// minimum length scale of the element update runs fused with Sync
// (k_min_length_scale_sync).
//
// Element kernels run one thread per tetrahedron: a warp holds three
// elements in lanes 0-9, 10-19, 20-29 (lanes 30-31 idle).  Element sums
// (volume, traces) are gathered lane by lane with shuffles and added in the
// reference's tet order, so they round like the reference's loops.  Node
// kernels run one thread per node and gather the 8 adjacent hexes x 5 tets in
// the reference's fixed order (Force.c:87-181): no atomics, bit-reproducible.
//
// Geometry (volumes, face areas and normals) is never stored: each kernel
// recomputes it from the coordinates with the reference's formulas, which
// gives the same bits the reference stored in its element structs.
#pragma once

#include <math_constants.h>

#include "snac_device.cuh"

namespace snac {

struct Mesh {
    int nx, ny, nz, nnx, nny, nnz;
    long long ne, nn;
    long long ner;  // row length of the tet-major per-tet arrays: ne rounded up to 4 (32-byte rows)
};

// Per-tet force and energy terms are stored tet-major, one row per
// (tet-in-hex, face, component) holding every element: entry (e, t, ...) sits
// at row(t, ...) * ner + e.  The element kernels write a row segment per
// group of elements, and the node gathers, which read a fixed (t, face) for
// consecutive elements along x, load consecutive addresses.

struct Fields {
    const double4* pos;      // current coordinates (x, y, z) and temperature (w)
    double4* pos_next;       // written by k_loop_nodes (coordinates are double-buffered)
    double4* vel;            // velocity (x, y, z) and temperature0 (w)
    double4* force;          // damped force (x, y, z) and inertial mass (w)
    double* stress;          // [ne*10][6]
    double* eps_p;           // [ne*10]  plastic strain (plastic, visco-plastic)
    double* pst;             // [ne*10][6] plastic strain tensor (visco-plastic with a Drucker-Prager phase)
    double* visc;            // [ne*10]  viscosity (visco-plastic, Maxwell)
    double* density;         // [ne*10]  only when some phase has alpha or beta != 0
    double* vol;             // [ne*10][2] volume, old volume (Maxwell)
    double* hflux;           // rows (t, 0..5): face energy terms (q.n A/6), Cp rho V/8, thermal stress
    double* tpre;            // [nn] temperature before the BCs (temperature + density)
    double* fterm;           // rows (t, face, xyz): stress.n.A/6 of each face (Force.c:154-165)
    double* fgrav;           // rows (t): g rho V / 8 (Force.c:173)
    double* fmass;           // rows (t, face) (constant dt) or (t): inertial-mass term (Force.c:107-140)
    const uchar4* bc;        // per node: velocity-VC index of x, y, z and temperature-VC index (255 = free)
    const double* vbc_val;   // [n_vc][3]
    const double* tbc_val;   // [n_tc]
    const unsigned char* mat;        // [ne] phase, NULL = 0
    const DevMaterial* mats;         // phase table of this model
    double* residual_fr;             // [nn] Winkler residual force of step 1 (winkler/Force.c:154-161)
    double* escal;                   // [ne][4] element strain rate, stress, hydroPressure, aps
                                     // (written on steps with sc->want_scalars; NULL = never)
    const double* coh_scale;         // [ne] or NULL
    const double* fric_scale;        // [ne] or NULL
    const double* visc_scale;        // [ne] or NULL
    DevScalars* sc;
};

#ifndef SNAC_VOLUME_ONLY
#define SNAC_VOLUME_ONLY 1
#endif
struct Config {
    int dt_type, constitutive, temperature, thermal_stress, has_density, time_step_zero;
    double gravity, demf;
    double strain_inert;
    int winkler;          // SnacWinklerForce on Snac_EP_Force
    int traction;         // SnacTractionBC on Snac_EP_Force (after Winkler)
    double topo_kappa, topo_crit;  // surface-topography diffusion
    double pisos, rzbo;   // its isostatic pressure and reference bottom depth
    int prefetch_ahead;   // element blocks resident at once (SMs x blocks per SM): the L2 prefetch distance
    // one phase, no density coupling, dynamic or wave dt: a tet's gravity and
    // inertial-mass terms are the same multiples of its volume for every tet,
    // so the element kernels store the volume alone (in the fgrav row) and
    // the node gather forms both terms from it with the same operations
    // (SNAC_VOLUME_ONLY = 0 turns this off, for measurement)
    int vonly;
    // phase 0, the only phase of a model without a per-element phase array:
    // the element kernels of such models read it from their parameters
    // (constant-bank operands) instead of loading it from the phase table
    DevMaterial m0;
};

#ifndef SNAC_ELEM_MINB
#define SNAC_ELEM_MINB 4  // resident blocks per SM asked of the compiler (register budget, measured best)
#endif
#ifndef SNAC_ELEM_WARPS
#define SNAC_ELEM_WARPS 4
#endif
constexpr int ELEM_WARPS = SNAC_ELEM_WARPS;    // warps per block in the element kernels
constexpr int ELEM_PER_BLOCK = ELEM_WARPS * 3;  // 12 elements per block
constexpr unsigned FULL = 0xffffffffu;
constexpr int HF_STRIDE = 6;  // per-tet heat record: 4 face energy terms, lumped capacity, thermal stress

__device__ __forceinline__ long long node_id(const Mesh& m, int i, int j, int k) {
    return (long long)i + (long long)j * m.nnx + (long long)k * m.nnx * m.nny;
}

// x = i + j a + k a b.  Index arithmetic in 32 bits whenever the index fits:
// a 64-bit integer division is a long software routine on the GPU, a 32-bit
// one a few instructions (the branch is uniform across a launch).
__device__ __forceinline__ void split3(long long x, int a, int b, int& i, int& j, int& k) {
    if (x >= 0 && x < 0x7fffffffLL) {
        const unsigned u = (unsigned)x, q = u / (unsigned)a, r = q / (unsigned)b;
        i = (int)(u - q * (unsigned)a);
        j = (int)(q - r * (unsigned)b);
        k = (int)r;
    } else {
        i = (int)(x % a);
        j = (int)((x / a) % b);
        k = (int)(x / ((long long)a * b));
    }
}

__device__ __forceinline__ void elem_ijk(const Mesh& m, long long e, int& i, int& j, int& k) {
    split3(e, m.nx, m.ny, i, j, k);
}

__device__ __forceinline__ long long corner_node(const Mesh& m, int i, int j, int k, int corner) {
    return node_id(m, i + corner_di(corner), j + corner_dj(corner), k + corner_dk(corner));
}

__device__ __forceinline__ int phase_of(const Fields& F, long long e) { return F.mat ? (int)F.mat[e] : 0; }

// The value of lane (base + u) of this lane's element group.
__device__ __forceinline__ double grp(double v, int base, int u) { return __shfl_sync(FULL, v, base + u); }

// Sum over the 10 tets of the group, added in tet order starting from 0.
__device__ __forceinline__ double grp_sum(double v, int base) {
    double s = 0.0f;
#pragma unroll
    for (int u = 0; u < NT; u++) s += grp(v, base, u);
    return s;
}

// a tet's six stress components as three 16-byte accesses (the [nq][6]
// rows start on 48-byte boundaries)
__device__ __forceinline__ void load_stress(const Fields& F, long long q, double st[6]) {
    const double2* p = reinterpret_cast<const double2*>(F.stress + q * 6);
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const double2 v = p[a];
        st[2 * a] = v.x;
        st[2 * a + 1] = v.y;
    }
}
__device__ __forceinline__ void store_stress(const Fields& F, long long q, const double st[6]) {
    double2* p = reinterpret_cast<double2*>(F.stress + q * 6);
#pragma unroll
    for (int a = 0; a < 3; a++) p[a] = make_double2(st[2 * a], st[2 * a + 1]);
}

struct TetSlot {
    int lane, base, t;
    long long e, q;
    bool active;
    int i, j, k;
};

__device__ __forceinline__ TetSlot tet_slot(const Mesh& m, int lb) {
    TetSlot s;
    s.lane = threadIdx.x & 31;
    int g = s.lane / 10;
    s.base = g * 10;
    s.t = s.lane - s.base;
    long long warp = (long long)lb * ELEM_WARPS + (threadIdx.x >> 5);
    s.e = warp * 3 + g;
    s.active = (g < 3) && (s.e < m.ne);
    if (g >= 3) {  // lanes 30, 31 mirror lane 0-9 group 0 slots so shuffles stay in range
        s.base = 0;
        s.t = s.lane - 30;
    }
    s.q = s.e * NT + s.t;
    if (s.active)
        elem_ijk(m, s.e, s.i, s.j, s.k);
    else
        s.i = s.j = s.k = 0;
    return s;
}

// loads the tet's 4 corners (coordinates, velocities, temperatures)
__device__ __forceinline__ void load_tet(const Mesh& m, const Fields& F, const TetSlot& s, V3 c[4], V3 v[4],
                                         double T[4], double T0[4]) {
#pragma unroll
    for (int qn = 0; qn < 4; qn++) {
        if (s.active) {
            long long n = corner_node(m, s.i, s.j, s.k, tet_node_rt(s.t, qn));
            double4 p = F.pos[n];
            double4 w = F.vel[n];
            c[qn] = {p.x, p.y, p.z};
            T[qn] = p.w;
            v[qn] = {w.x, w.y, w.z};
            T0[qn] = w.w;
        } else {  // a regular dummy tet keeps inactive lanes finite
            c[qn] = {qn == 1 ? 1.0 : 0.0, qn == 2 ? 1.0 : 0.0, qn == 3 ? 1.0 : 0.0};
            v[qn] = {0.0, 0.0, 0.0};
            T[qn] = T0[qn] = 0.0;
        }
    }
}

// What the constitutive update reads from global memory besides the
// corners and the stress.  The face stash below is a compiler barrier, so
// these loads stay after it; so that they do not wait a full memory round
// trip in the middle of the tet's arithmetic, the element kernels prefetch
// their lines into L1 at the start (prefetch_tet_in), which costs no
// registers (loading the values that early would hold them across the
// geometry, where registers are scarcest, and made the visco-plastic
// instances spill).
struct TetIn {
    double eps_p;                 // plastic strain (plastic, visco-plastic)
    double coh, fric, visc;       // per-element parameter scales (1 without them)
    double pst[6];                // plastic strain tensor (Drucker-Prager instances)
};

template <int PLUGIN>
__device__ __forceinline__ TetIn load_tet_in(const Fields& F, const TetSlot& s) {
    TetIn in;
    in.eps_p = 0.0;
    if (PLUGIN == SNAC_RHEOLOGY_PLASTIC || is_vp(PLUGIN))
        in.eps_p = s.active ? F.eps_p[s.q] : 0.0;
    for (int a = 0; a < 6; a++) in.pst[a] = 0.0;
    if (PLUGIN == SNAC_VP_DP && s.active) {
        const double2* p = reinterpret_cast<const double2*>(F.pst + s.q * 6);
        for (int a = 0; a < 3; a++) {
            const double2 w = p[a];
            in.pst[2 * a] = w.x;
            in.pst[2 * a + 1] = w.y;
        }
    }
    in.coh = (F.coh_scale && s.active) ? F.coh_scale[s.e] : 1.0;
    in.fric = (F.fric_scale && s.active) ? F.fric_scale[s.e] : 1.0;
    in.visc = (F.visc_scale && s.active) ? F.visc_scale[s.e] : 1.0;
    return in;
}

__device__ __forceinline__ void prefetch_l1(const void* p) { asm volatile("prefetch.global.L1 [%0];" ::"l"(p)); }

template <int PLUGIN>
__device__ __forceinline__ void prefetch_tet_in(const Fields& F, const TetSlot& s) {
    if (!s.active) return;
    if (PLUGIN == SNAC_RHEOLOGY_PLASTIC || is_vp(PLUGIN)) prefetch_l1(F.eps_p + s.q);
    if (PLUGIN == SNAC_VP_DP) prefetch_l1(F.pst + s.q * 6);
    if (s.t == 0) {  // one lane per hex for the per-element rows
        if (F.coh_scale) prefetch_l1(F.coh_scale + s.e);
        if (F.fric_scale) prefetch_l1(F.fric_scale + s.e);
        if (F.visc_scale) prefetch_l1(F.visc_scale + s.e);
    }
}

// ======================================================================================
// Snac_EP_CalcStresses: StrainRate.c:49-305, Stress.c:53-172 and the constitutive hook
// ======================================================================================
// st holds the tet's stress on entry (already rotated when fused with the
// element update); the new stress, plastic strain, viscosity, density and
// the Force terms are stored.
// The tet's four face areas and normals are needed again only by the force
// terms at the end of the stress update; across the constitutive update
// (the eigen-solve of a yielding tet needs ~60 registers) they wait in
// shared memory, one 16-double column per thread, instead of in registers
// that the compiler would otherwise spill to local memory.
__shared__ double face_stash[16 * ELEM_WARPS * 32];

__device__ __forceinline__ void stash_faces(const TetGeom& g) {
    constexpr int W = ELEM_WARPS * 32;
    const int tid = threadIdx.x;
#pragma unroll
    for (int f = 0; f < 4; f++) {
        face_stash[(f * 4 + 0) * W + tid] = g.A[f];
        face_stash[(f * 4 + 1) * W + tid] = g.n[f].x;
        face_stash[(f * 4 + 2) * W + tid] = g.n[f].y;
        face_stash[(f * 4 + 3) * W + tid] = g.n[f].z;
    }
    asm volatile("" ::: "memory");  // keep the copies in shared memory, not in registers
}
__device__ __forceinline__ void unstash_faces(TetGeom& g) {
    constexpr int W = ELEM_WARPS * 32;
    const int tid = threadIdx.x;
    asm volatile("" ::: "memory");
#pragma unroll
    for (int f = 0; f < 4; f++) {
        g.A[f] = face_stash[(f * 4 + 0) * W + tid];
        g.n[f].x = face_stash[(f * 4 + 1) * W + tid];
        g.n[f].y = face_stash[(f * 4 + 2) * W + tid];
        g.n[f].z = face_stash[(f * 4 + 3) * W + tid];
    }
}

template <int PLUGIN, bool ONE>
__device__ __forceinline__ void stress_update(const Mesh& m, const Fields& F, const Config& cfg, const TetSlot& s,
                                              const V3 v[4], const double T[4], const TetGeom& g, double st[6],
                                              const double dt, const double* sr_given = nullptr) {
    double sr[6];
    if (sr_given) {  // the fused kernel formed it with the spin rates
#pragma unroll
        for (int a = 0; a < 6; a++) sr[a] = sr_given[a];
    } else {
        tet_strain_rate(v, g, sr);
    }

    // element volume: UpdateElement.c:141,267 then 2*volume (StrainRate.c:62)
    double vsum = grp_sum(g.V, s.base);
    double elemVolume = 2.0 * (vsum * 0.5);
    // mixed discretisation, StrainRate.c:272-289
    double trace = dv3(sr[0] + sr[1] + sr[2]);
    // each term trace_u * V_u is formed on its own lane and gathered (the same
    // product the sum would form from the two gathered factors)
    const double traceV = trace * g.V;
    double partial = 0.0f;
#pragma unroll
    for (int u = 0; u < NT; u++) partial += grp(traceV, s.base, u);
    const double zE = recip(elemVolume);
    double corr = -1.0f * trace + dvz(partial, elemVolume, zE);
    sr[0] += corr;
    sr[1] += corr;
    sr[2] += corr;
    // scalar element outputs for the dump writers, on the steps that need them
    const bool want = F.escal != nullptr && F.sc->want_scalars;
    if (want) {
        // StrainRate.c:284-304
        double srVolAvg = grp_sum(sr[1] * sr[2] + sr[2] * sr[0] + sr[0] * sr[1], s.base);
        double srOtherAvg = grp_sum(sr[3] * sr[3] + sr[5] * sr[5] + sr[4] * sr[4], s.base);
        srVolAvg = dv10(srVolAvg);
        srOtherAvg = dv10(srOtherAvg);
        if (s.active && s.t == 0) F.escal[s.e * 4 + 0] = 0.5f * sqrt(0.5f * fabs(-1.0f * srVolAvg + srOtherAvg));
    }

    // strain, Stress.c:71-82
    double e[6];
#pragma unroll
    for (int a = 0; a < 6; a++) e[a] = sr[a] * dt;

    stash_faces(g);
    const TetIn in = load_tet_in<PLUGIN>(F, s);
    const int ph = s.active ? phase_of(F, s.e) : 0;
    const DevMaterial& M = ONE ? cfg.m0 : F.mats[ph];  // ONE: the model has one phase
    double eps_p = in.eps_p, eta = 0.0;
    // what the Drucker-Prager return map needs from the viscous update
    double dp_sd[3] = {0.0, 0.0, 0.0}, dp_S0[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    double dp_vic1 = 0.0, dp_vic2 = 0.0, dp_bulkm = 0.0;

    double sp[3] = {0, 0, 0}, cn[3][3];
    // softening-table lookup results of this tet (for the carry-over between tets)
    double fa = 0.0f, da = 0.0f, co = 0.0f, hd = 0.0f;
    int matched = 0;

    if (PLUGIN == SNAC_RHEOLOGY_ELASTIC) {
        // elastic/Constitutive.c:40-66
        const double a2 = M.lambda;
        const double sh2 = 2.0 * M.mu;
        double tr = e[0] + e[1] + e[2];
        st[0] += sh2 * e[0] + a2 * (tr);
        st[1] += sh2 * e[1] + a2 * (tr);
        st[2] += sh2 * e[2] + a2 * (tr);
        st[3] += sh2 * e[3];
        st[4] += sh2 * e[4];
        st[5] += sh2 * e[5];
    } else if (PLUGIN == SNAC_RHEOLOGY_MAXWELL) {
        // maxwell/Constitutive.c:47-184
        const double bulkm = M.lambda + dv3(2.0f * M.mu);
        double vold = s.active ? F.vol[s.q * 2 + 1] : 1.0;
        double vcur = s.active ? F.vol[s.q * 2 + 0] : 1.0;
        double trace_stress = st[0] + st[1] + st[2];
        double trace_strain = dv(vcur, vold) - 1.0f;
        double straind[3], stressd[3];
        const double tn3 = dv3(trace_strain), ts3 = dv3(trace_stress);
        for (int a = 0; a < 3; a++) straind[a] = e[a] - tn3;
        for (int a = 0; a < 3; a++) stressd[a] = st[a] - ts3;
        double srJ2 = sqrt(fabs(straind[1] * straind[2] + straind[2] * straind[0] + straind[0] * straind[1] -
                                e[3] * e[3] - e[4] * e[4] - e[5] * e[5])) /
                      dt;
        if (srJ2 == 0.0f) srJ2 = M.refsrate;
        double avgTemp = 0.0;
        for (int qn = 0; qn < 4; qn++) avgTemp += 0.25 * T[qn];
        eta = arrhenius_viscosity(M, M.refvisc, srJ2, avgTemp);
        if (s.active && !isfinite(eta)) report(F.sc, SNAC_GPU_ENAN, s.e);
        if (ph == 0) maxwell_update(st, e, stressd, straind, ts3, trace_strain, M.mu, eta, dt, bulkm);
    } else {
        if (PLUGIN == SNAC_RHEOLOGY_PLASTIC) {
            // elastic trial, plastic/Constitutive.c:114-121
            double tr = e[0] + e[1] + e[2];
            st[0] += (2.0f * M.mu) * e[0] + M.lambda * (tr);
            st[1] += (2.0f * M.mu) * e[1] + M.lambda * (tr);
            st[2] += (2.0f * M.mu) * e[2] + M.lambda * (tr);
            st[3] += (2.0f * M.mu) * e[3];
            st[4] += (2.0f * M.mu) * e[4];
            st[5] += (2.0f * M.mu) * e[5];
            if (s.active && M.plstrain[0] != 0.0) report(F.sc, SNAC_GPU_EINVAL, s.e);
        } else {
            // visco-plastic Maxwell step, viscoplastic/Constitutive.c:158-257
            const double bulkm = M.lambda + dv3(2.0f * M.mu);
            if (cfg.thermal_stress) {
                double ts = s.active ? F.hflux[(long long)(s.t * HF_STRIDE + 5) * m.ner + s.e] : 0.0;
                st[0] += ts;
                st[1] += ts;
                st[2] += ts;
            }
            if (PLUGIN == SNAC_VP_DP)  // Stress0, viscoplastic/Constitutive.c:165-170
                for (int a = 0; a < 6; a++) dp_S0[a] = st[a];
            double trace_stress = st[0] + st[1] + st[2];
            double trace_strain = e[0] + e[1] + e[2];
            double straind[3], stressd[3];
            const double tn3 = dv3(trace_strain), ts3 = dv3(trace_stress);
            for (int a = 0; a < 3; a++) straind[a] = e[a] - tn3;
            for (int a = 0; a < 3; a++) stressd[a] = st[a] - ts3;
            // viscoplastic/Constitutive.c:189 reads strain[1][0], strain[2][0] and stress[2][0]
            // (the pointer, not the tensor, is indexed); those entries are always zero.
            const double lower = 0.0;
            double srJ2 = sqrt(fabs(straind[1] * straind[2] + straind[2] * straind[0] + straind[0] * straind[1] -
                                    (lower) * (lower) - (lower) * (lower) - (lower) * (lower))) /
                          dt;
            if (srJ2 == 0.0f) srJ2 = M.refsrate;
            double avgTemp = 0.0;
            for (int qn = 0; qn < 4; qn++) avgTemp += 0.25 * T[qn];
            double refvisc = M.refvisc;
            if (F.visc_scale && s.active) refvisc = M.refvisc * in.visc;
            eta = arrhenius_viscosity(M, refvisc, srJ2, avgTemp);
            if (s.active && !isfinite(eta)) report(F.sc, SNAC_GPU_ENAN, s.e);
            maxwell_update(st, e, stressd, straind, ts3, trace_strain, M.mu, eta, dt, bulkm, dp_vic1, dp_vic2);
            if (PLUGIN == SNAC_VP_DP) {
                for (int a = 0; a < 3; a++) dp_sd[a] = stressd[a];
                dp_bulkm = bulkm;
            }
        }
        // piecewise-linear softening (plastic/Constitutive.c:133-159 with break and
        // clamp; viscoplastic/Constitutive.c:279-293 without either: the last
        // matching segment wins)
        const double cs = in.coh;
        const double fsc = in.fric;
        for (int i = 0; i < M.nsegments; i++) {
            const double pl1 = M.plstrain[i];
            const double pl2 = M.plstrain[i + 1];
            double f0 = F.fric_scale ? M.fric[i] * fsc : M.fric[i];
            double f1 = F.fric_scale ? M.fric[i + 1] * fsc : M.fric[i + 1];
            double c0 = F.coh_scale ? M.coh[i] * cs : M.coh[i];
            double c1 = F.coh_scale ? M.coh[i + 1] * cs : M.coh[i + 1];
            if (eps_p >= pl1 && eps_p <= pl2) {
                const double dpl = pl2 - pl1, zpl = M.zpl[i];  // = RN(1 / dpl)
                double tg[3] = {f1 - f0, M.dil[i + 1] - M.dil[i], c1 - c0};
                dvz_n(tg, dpl, zpl);
                const double tgf = tg[0], tgd = tg[1], tgc = tg[2];
                fa = f0 + tgf * (eps_p - pl1);
                da = M.dil[i] + tgd * (eps_p - pl1);
                co = c0 + tgc * (eps_p - pl1);
                hd = tgc;
                matched = 1;
                if (PLUGIN == SNAC_RHEOLOGY_PLASTIC) break;
            } else if (PLUGIN == SNAC_RHEOLOGY_PLASTIC && i == M.nsegments - 1 && eps_p > pl2) {
                fa = F.fric_scale ? M.fric[M.nsegments] * fsc : M.fric[M.nsegments];
                da = M.dil[M.nsegments];
                co = F.coh_scale ? M.coh[M.nsegments] * cs : M.coh[M.nsegments];
                hd = 0.0;
                matched = 1;
                break;
            }
        }
    }

    double pst[6];
    for (int a = 0; a < 6; a++) pst[a] = in.pst[a];
    if (PLUGIN == SNAC_RHEOLOGY_PLASTIC || is_vp(PLUGIN)) {
        // The reference keeps the table values (and the tension cutoff) in
        // variables that outlive the tet loop: a tet whose lookup matched no
        // segment reuses the previous tet's values, 0 before the first match.
        double frictionAngle = fa, dilationAngle = da, cohesion = co, hardening = hd;
        // warp-uniform test: when every tet of the warp matched, each uses its own values
        if (__ballot_sync(FULL, s.active && !matched) != 0u) {
            unsigned mb = __ballot_sync(FULL, matched && s.active);
            unsigned mine = (mb >> s.base) & ((1u << (s.t + 1)) - 1u);
            int src = mine ? (31 - __clz(mine)) : -1;
            double src_fa = __shfl_sync(FULL, fa, s.base + (src < 0 ? 0 : src));
            double src_da = __shfl_sync(FULL, da, s.base + (src < 0 ? 0 : src));
            double src_co = __shfl_sync(FULL, co, s.base + (src < 0 ? 0 : src));
            double src_hd = __shfl_sync(FULL, hd, s.base + (src < 0 ? 0 : src));
            frictionAngle = src < 0 ? 0.0f : src_fa;
            dilationAngle = src < 0 ? 0.0f : src_da;
            cohesion = src < 0 ? 0.0f : src_co;
            hardening = src < 0 ? 0.0f : src_hd;
        }
        // tension cutoff st = min(ten_off, c / tan(phi)) when phi > 0, else carried over
        const bool fconst = M.fric_const && frictionAngle == M.fric0;
        bool phi_ok = (PLUGIN == SNAC_RHEOLOGY_PLASTIC) ? (frictionAngle >= 0.0f) : (frictionAngle > 0.0f);
        double st_own = 0.0;
        if (phi_ok) {
            st_own = M.ten_off;
            if (frictionAngle > 0.0) {
                double tmp = fconst ? dvz(cohesion, M.tan_fric0, M.ztan_fric0) : dv(cohesion, tan_fric(M, frictionAngle));
                if (tmp < st_own) st_own = tmp;
            }
        }
        double stc = st_own;
        if (__ballot_sync(FULL, s.active && !phi_ok) != 0u) {
            unsigned pb = __ballot_sync(FULL, phi_ok && s.active);
            unsigned pm = (pb >> s.base) & ((1u << (s.t + 1)) - 1u);
            int psrc = pm ? (31 - __clz(pm)) : -1;
            double st_c = __shfl_sync(FULL, st_own, s.base + (psrc < 0 ? 0 : psrc));
            stc = psrc < 0 ? 0.0 : st_c;
        }
        if (PLUGIN == SNAC_RHEOLOGY_PLASTIC && s.active && frictionAngle < 0.0f)
            report(F.sc, SNAC_GPU_EPHYSICS, s.e);  // plastic/Constitutive.c:175 abort()
        if (PLUGIN == SNAC_VP_DP && !M.yield_mc) {
            // viscoplastic/Constitutive.c:372-518 (the principal stresses the
            // reference computes first are not used by this branch)
            if (s.active)
                dp_return_map(st, dp_sd, dp_S0, e, dp_vic1, dp_vic2, M.mu, dp_bulkm, tan_fric(M, frictionAngle),
                              tan_dil(M, dilationAngle), cohesion, stc, M.dp_tol, M.dp_maxit, pst, eps_p);
        } else {
            double sphi = sin_fric(M, frictionAngle);
            double spsi = sin_dil(M, dilationAngle);
            double anphi = fconst ? M.anphi0 : dv(1.0f + sphi, 1.0f - sphi);
            double anpsi = (M.dil_const && dilationAngle == M.dil0) ? M.anpsi0 : dv(1.0f + spsi, 1.0f - spsi);
            const double a1 = M.lambda + 2.0f * M.mu;
            const double a2 = M.lambda;
            // The reference always computes the principal stresses; they only
            // matter when the tet yields.  A tet that provably stays inside the
            // yield surface keeps its trial stress without the eigen-solve.
            if (!surely_elastic(st, cohesion, anphi, fconst ? M.sq_anphi0 : sqrt(anphi), stc)) {
                principal_stresses(st, sp, cn);
                mc_return_map(sp, cn, st, eps_p, cohesion, hardening, anphi, anpsi, stc, a1, a2);
            }
        }
    }

    // trace averaging over the 10 tets, Stress.c:87-137
    double traceS = dv3(st[0] + st[1] + st[2]);
    const double traceSV = traceS * g.V;
    double partialS = 0.0f;
#pragma unroll
    for (int u = 0; u < NT; u++) partialS += grp(traceSV, s.base, u);
    const double avgTrace = dvz(partialS, elemVolume, zE);
    double cs2 = -1.0f * traceS + avgTrace;
    st[0] += cs2;
    st[1] += cs2;
    st[2] += cs2;
    if (want) {
        // Stress.c:130-156: the element's scalar stress and hydrostatic pressure
        double sVolAvg = grp_sum((st[1] - avgTrace) * (st[2] - avgTrace) + (st[2] - avgTrace) * (st[0] - avgTrace) +
                                     (st[0] - avgTrace) * (st[1] - avgTrace),
                                 s.base);
        double sOtherAvg = grp_sum(st[3] * st[3] + st[5] * st[5] + st[4] * st[4], s.base);
        double pressure = grp_sum(dv3(st[0] + st[1] + st[2]), s.base);
        sVolAvg = dv10(sVolAvg);
        sOtherAvg = dv10(sOtherAvg);
        pressure = dv10(pressure);
        // plastic/Constitutive.c:239-244, viscoplastic/Constitutive.c:519-523: aps
        double aps = 0.0;
        if (PLUGIN == SNAC_RHEOLOGY_PLASTIC || is_vp(PLUGIN))
            aps = dv(grp_sum(eps_p * g.V, s.base), vsum);
        if (s.active && s.t == 0) {
            F.escal[s.e * 4 + 1] = 0.5f * sqrt(0.5f * fabs(-1.0f * sVolAvg + sOtherAvg));
            F.escal[s.e * 4 + 2] = -1.0 * pressure;
            F.escal[s.e * 4 + 3] = aps;
        }
    }

    if (cfg.has_density) {
        // Stress.c:125-170: pressure = mean tet trace/3, density update
        double ptet = dv3(st[0] + st[1] + st[2]);
        double pressure = 0.0f;
#pragma unroll
        for (int u = 0; u < NT; u++) pressure += grp(ptet, s.base, u);
        pressure = dv10(pressure);
        double avgT = 0.0;
        if (cfg.temperature) {
            // UpdateAverageTemp_LoopElements (Heat.c:143-172) ran before the
            // temperature BCs were re-applied: use the pre-BC temperatures
            avgT = 0.0;
            int ei = 0, ej = 0, ek = 0;  // recomputed here: the slot's i, j, k need not stay live
            if (s.active) elem_ijk(m, s.e, ei, ej, ek);
            for (int qn = 0; qn < 4; qn++) {
                long long n = s.active ? corner_node(m, ei, ej, ek, tet_node_rt(s.t, qn)) : 0;
                avgT += F.tpre[n] / (1.0f * 4);
            }
        }
        if (s.active) F.density[s.q] = M.density * (1.0 - M.alpha * (avgT - M.reftemp) + M.beta * pressure);
    }

    // Per-tet terms of Snac_Force (Force.c:107-180), evaluated here where the
    // tet's geometry and new stress already are.  k_loop_nodes adds them in
    // the reference's node-centred order, so the sums keep their bits.
    TetGeom gf;  // the faces back from shared memory
    gf.V = g.V;
    gf.zV = g.zV;
    unstash_faces(gf);
    if (s.active) {
        const double rho = cfg.has_density ? F.density[s.q] : M.density;
        const long long R = m.ner;
        double* o = F.fterm + (long long)(s.t * 12) * R + s.e;  // rows (t, face, component)
#pragma unroll
        for (int f = 0; f < 4; f++) {
            const V3& nr = gf.n[f];
            const double A = gf.A[f];
            double t[3] = {(st[0] * nr.x + st[3] * nr.y + st[4] * nr.z) * A, (st[3] * nr.x + st[1] * nr.y + st[5] * nr.z) * A,
                           (st[4] * nr.x + st[5] * nr.y + st[2] * nr.z) * A};
            dvk_n(t, 6.0, Z6);
            o[(f * 3 + 0) * R] = t[0];
            o[(f * 3 + 1) * R] = t[1];
            o[(f * 3 + 2) * R] = t[2];
        }
        const long long qt = (long long)s.t * R + s.e;  // row t
        const double factor4 = 1.0f / 4.0f;
        if (ONE && cfg.vonly) {
            F.fgrav[qt] = gf.V;
        } else {
            F.fgrav[qt] = cfg.gravity * rho * gf.V * 0.125;  // x * 2^-3 rounds as x / 8
        }
        if (ONE && cfg.vonly) {
            // both terms formed by the node gather
        } else if (cfg.dt_type == SNAC_DT_DYNAMIC) {
            const double sos = F.sc->speed_of_sound;
            const double inertialDensity = ONE ? F.sc->inertial_density0 : dv(M.lambda + 2.0f * M.mu, sos * sos);
            F.fmass[qt] = factor4 * inertialDensity * gf.V;
        } else if (cfg.dt_type == SNAC_DT_CONSTANT) {
            const double alpha1 = (M.lambda + 2.0f * M.mu);
            const double nineV = 9.0f * gf.V, z9V = recip(nineV);
#pragma unroll
            for (int f = 0; f < 4; f++) {
                const V3& nr = gf.n[f];
                const double A = gf.A[f];
                double area_sum = 0.0, temp;
                temp = (nr.x * A) * (nr.x * A);
                if (temp > area_sum) area_sum = temp;
                temp = (nr.y * A) * (nr.y * A);
                if (temp > area_sum) area_sum = temp;
                temp = (nr.z * A) * (nr.z * A);
                if (temp > area_sum) area_sum = temp;
                F.fmass[(long long)(s.t * 4 + f) * R + s.e] = dvz(alpha1 * area_sum, nineV, z9V) * (dt * dt);
            }
        } else {
            F.fmass[qt] = factor4 * rho * gf.V;
        }
    }

    if (s.active) {
        store_stress(F, s.q, st);
        bool ok = true;
#pragma unroll
        for (int a = 0; a < 6; a++) ok = ok & (bool)isfinite(st[a]);
        if (!ok) report(F.sc, SNAC_GPU_ENAN, s.e);  // Stress.c:161-166
        if (PLUGIN == SNAC_RHEOLOGY_PLASTIC || is_vp(PLUGIN)) F.eps_p[s.q] = eps_p;
        if (is_vp(PLUGIN) || (PLUGIN == SNAC_RHEOLOGY_MAXWELL && ph == 0)) F.visc[s.q] = eta;
        if (PLUGIN == SNAC_VP_DP) {
            double2* p = reinterpret_cast<double2*>(F.pst + s.q * 6);
            for (int a = 0; a < 3; a++) p[a] = make_double2(pst[2 * a], pst[2 * a + 1]);
        }
    }
}

template <int PLUGIN, bool ONE>
__device__ __forceinline__ void k_calc_stresses_body(const Mesh& m, const Fields& F, const Config& cfg, int lb) {
    TetSlot s = tet_slot(m, lb);
    prefetch_tet_in<PLUGIN>(F, s);
    V3 c[4], v[4];
    double T[4], T0[4];
    load_tet(m, F, s, c, v, T, T0);
    TetGeom g;
    tet_geometry(c, g);
    double st[6] = {0, 0, 0, 0, 0, 0};
    if (s.active) {
        load_stress(F, s.q, st);
    }
    stress_update<PLUGIN, ONE>(m, F, cfg, s, v, T, g, st, F.sc->dt);
}

template <int PLUGIN, bool ONE>
__global__ void __launch_bounds__(ELEM_WARPS * 32, SNAC_ELEM_MINB) k_calc_stresses(Mesh m, Fields F, Config cfg) {
    k_calc_stresses_body<PLUGIN, ONE>(m, F, cfg, blockIdx.x);
}

// UpdateElement.c:84-91 volume bookkeeping (Maxwell reads V/V_old) and the
// Jaumann rotation of the stress (:145-265) of one tet; returns the rotated stress.
#ifndef SNAC_SHARED_SUMS
#define SNAC_SHARED_SUMS 0
#endif
// UpdateElement.c:84-91 volume bookkeeping and the Jaumann rotation with
// given spin rates
template <int PLUGIN>
__device__ __forceinline__ void element_update_tet_by(const Fields& F, const Config& cfg, const TetSlot& s,
                                                      const TetGeom& g, const double (&r)[3], double dt, double st[6]) {
    if (PLUGIN == SNAC_RHEOLOGY_MAXWELL && s.active) {
        double vc = F.vol[s.q * 2 + 0];
        F.vol[s.q * 2 + 1] = cfg.time_step_zero ? g.V : vc;
        F.vol[s.q * 2 + 0] = g.V;
    }
    if (s.active) {
        load_stress(F, s.q, st);
        rotate_stress_by(r, dt, st);
    }
}

template <int PLUGIN>
__device__ __forceinline__ void element_update_tet(const Fields& F, const Config& cfg, const TetSlot& s, const V3 v[4],
                                                   const TetGeom& g, double dt, double st[6]) {
    if (PLUGIN == SNAC_RHEOLOGY_MAXWELL && s.active) {
        double vc = F.vol[s.q * 2 + 0];
        F.vol[s.q * 2 + 1] = cfg.time_step_zero ? g.V : vc;
        F.vol[s.q * 2 + 0] = g.V;
    }
    if (s.active) {
        load_stress(F, s.q, st);
        rotate_stress(v, g, dt, st);
    }
}

// The end of step n (element update with dt_n, whose geometry and velocities
// are already final) fused with the stress update of step n+1 (dt_{n+1},
// same geometry and velocities): one geometry evaluation, one stress
// read-modify-write.  Used when no energy hook sits between the two.
template <int PLUGIN, bool ONE>
__device__ __forceinline__ void k_fused_step_body(const Mesh& m, const Fields& F, const Config& cfg, int lb,
                                                  bool count_step = true) {
    TetSlot s = tet_slot(m, lb);
    prefetch_tet_in<PLUGIN>(F, s);
    if (count_step && lb == 0 && threadIdx.x == 0) {  // _AbstractContext_Execute_Hook: timeStep++, currentTime += dt
        F.sc->time_step += 1;
        F.sc->current_time += F.sc->dt;
    }
    V3 c[4], v[4];
    double T[4], T0[4];
    load_tet(m, F, s, c, v, T, T0);
    TetGeom g;
    tet_geometry(c, g);
    double st[6] = {0, 0, 0, 0, 0, 0};
#if SNAC_SHARED_SUMS
    double r[3], sr[6];
    spin_and_strain_rates(v, g, r, sr);
    element_update_tet_by<PLUGIN>(F, cfg, s, g, r, F.sc->dt_rot, st);
    stress_update<PLUGIN, ONE>(m, F, cfg, s, v, T, g, st, F.sc->dt, sr);
#else
    element_update_tet<PLUGIN>(F, cfg, s, v, g, F.sc->dt_rot, st);
    stress_update<PLUGIN, ONE>(m, F, cfg, s, v, T, g, st, F.sc->dt);
#endif
}

#ifndef SNAC_L2_PREFETCH
#define SNAC_L2_PREFETCH 0
#endif
// L2 prefetch of what element block `blk` will read (the block one wave of
// resident blocks later): the corner nodes of its hexes, one (hex, corner)
// per thread, and its stress, plastic-strain and cohesion-scale rows as bulk
// prefetches.  Every address lies inside its array (hexes < ne, nodes of
// those hexes) and the bulk ranges start on 16-byte boundaries and are
// multiples of 16 bytes (480 and 80 bytes per hex; the 8-byte scale rows are
// rounded down).  A prefetch changes no value.
__device__ __forceinline__ void prefetch_block(const Mesh& m, const Fields& F, long long blk) {
    const long long e0 = blk * ELEM_PER_BLOCK;
    if (e0 >= m.ne) return;
    const int nh = (int)((m.ne - e0) < ELEM_PER_BLOCK ? (m.ne - e0) : ELEM_PER_BLOCK);
    const int t = threadIdx.x;
    if (t < nh * 8) {
        int i, j, k;
        elem_ijk(m, e0 + t / 8, i, j, k);
        const long long n = corner_node(m, i, j, k, t % 8);
        asm volatile("prefetch.global.L2 [%0];" ::"l"(F.pos + n));
        asm volatile("prefetch.global.L2 [%0];" ::"l"(F.vel + n));
    } else if (t == ELEM_WARPS * 32 - 1) {
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(F.stress + e0 * NT * 6), "r"(nh * NT * 48));
    } else if (t == ELEM_WARPS * 32 - 2 && F.eps_p) {
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(F.eps_p + e0 * NT), "r"(nh * NT * 8));
    } else if (t == ELEM_WARPS * 32 - 3 && F.coh_scale && (nh * 8) / 16 > 0) {
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(F.coh_scale + e0), "r"((nh * 8) / 16 * 16));
    }
}

template <int PLUGIN, bool ONE>
__global__ void __launch_bounds__(ELEM_WARPS * 32, SNAC_ELEM_MINB) k_fused_step(Mesh m, Fields F, Config cfg) {
#if SNAC_L2_PREFETCH
    if (cfg.prefetch_ahead > 0) prefetch_block(m, F, (long long)blockIdx.x + cfg.prefetch_ahead);
#endif
    k_fused_step_body<PLUGIN, ONE>(m, F, cfg, blockIdx.x);
}

// Temperature runs: the element update of step n is deferred past the heat
// flux and temperature update of step n+1 (neither reads the stress) into
// the stress kernel of step n+1, which recomputes the same geometry anyway;
// the step counters were advanced by the heat-flux kernel.
template <int PLUGIN, bool ONE>
__global__ void __launch_bounds__(ELEM_WARPS * 32, SNAC_ELEM_MINB) k_fused_stress(Mesh m, Fields F, Config cfg) {
    k_fused_step_body<PLUGIN, ONE>(m, F, cfg, blockIdx.x, false);
}

// ======================================================================================
// Snac_EP_LoopElementsMomentum: UpdateElement.c:54-269 and the minLengthScale
// reduction of _Snac_Context_LoopElements (Context.c:1156-1184)
// ======================================================================================
template <int PLUGIN>
__device__ __forceinline__ void k_update_elements_body(const Mesh& m, const Fields& F, const Config& cfg,
                                                                                     int pending, int lb) {
    TetSlot s = tet_slot(m, lb);
    V3 c[4], v[4];
    double T[4], T0[4];
    load_tet(m, F, s, c, v, T, T0);
    TetGeom g;
    tet_geometry(c, g);
    double st[6];
    element_update_tet<PLUGIN>(F, cfg, s, v, g, pending ? F.sc->dt_rot : F.sc->dt, st);
    if (s.active) {
        store_stress(F, s.q, st);
    }
    if (pending) return;  // the minimum length scale of this geometry is already known
    double ls = 1.0e+27f;
#pragma unroll
    for (int f = 0; f < 4; f++) {
        double l = g.A[f];
        if (l) {
            l = fabs(dv(g.V, l));
            if (ls > l) ls = l;
        }
    }
    if (!s.active) ls = 1.0e+27f;
    if (s.active && g.V == 0.0) report(F.sc, SNAC_GPU_EVOLUME, s.e);
    // global minimum (exact: min does not round)
    for (int o = 16; o > 0; o >>= 1) ls = fmin(ls, __shfl_xor_sync(FULL, ls, o));
    if ((threadIdx.x & 31) == 0) atomicMin(&F.sc->minls_bits, (unsigned long long)__double_as_longlong(ls));
}

template <int PLUGIN>
__global__ void __launch_bounds__(ELEM_WARPS * 32, SNAC_ELEM_MINB) k_update_elements(Mesh m, Fields F, Config cfg,
                                                                                     int pending) {
    k_update_elements_body<PLUGIN>(m, F, cfg, pending, blockIdx.x);
}

// The minimum over all tets and faces of |V/A| (UpdateElement.c:109-139) for
// the current coordinates, without the rest of the element update.  For a
// tet, min_f RN(V/A_f) = RN(V / max_f A_f) because correctly rounded
// division is monotonic, and max_f A_f = RN(sqrt(max_f s_f))/2 for the same
// reason; faces with A = 0 are skipped as in the reference.
__device__ __forceinline__ double hex_min_length_scale(const Mesh& m, const Fields& F, int lb) {
    long long e = (long long)lb * blockDim.x + threadIdx.x;
    double ls = 1.0e+27f;
    if (e < m.ne) {
        int i, j, k;
        elem_ijk(m, e, i, j, k);
        V3 corner[8];
#pragma unroll
        for (int cc = 0; cc < 8; cc++) {
            double4 p = F.pos[corner_node(m, i, j, k, cc)];
            corner[cc] = {p.x, p.y, p.z};
        }
#pragma unroll
        for (int t = 0; t < NT; t++) {
            V3 c[4];
#pragma unroll
            for (int qn = 0; qn < 4; qn++) c[qn] = corner[tet_node(t, qn)];
            double V = tet_volume(c[0], c[1], c[2], c[3]);
            double smax = 0.0;
#pragma unroll
            for (int f = 0; f < 4; f++) {
                const V3 &c1 = c[face_node(f, 0)], &c2 = c[face_node(f, 1)], &c3 = c[face_node(f, 2)];
                double x2 = c2.x - c1.x, y2 = c2.y - c1.y, z2 = c2.z - c1.z;
                double x3 = c3.x - c1.x, y3 = c3.y - c1.y, z3 = c3.z - c1.z;
                double a = y2 * z3 - z2 * y3;
                double b = z2 * x3 - x2 * z3;
                double cc = x2 * y3 - y2 * x3;
                double sq = a * a + b * b + cc * cc;
                if (sq > smax) smax = sq;
            }
            double A = sqrt(smax) * 0.5;  // rounds as / 2
            if (A) {
                double l = fabs(dv(V, A));
                if (ls > l) ls = l;
            }
            if (V == 0.0) report(F.sc, SNAC_GPU_EVOLUME, e);
        }
    }
    return ls;
}

__device__ __forceinline__ void k_min_length_scale_body(const Mesh& m, const Fields& F, int lb) {
    double ls = hex_min_length_scale(m, F, lb);
    for (int o = 16; o > 0; o >>= 1) ls = fmin(ls, __shfl_xor_sync(FULL, ls, o));
    if ((threadIdx.x & 31) == 0) atomicMin(&F.sc->minls_bits, (unsigned long long)__double_as_longlong(ls));
}


// ======================================================================================
// Snac_EP_LoopNodesMomentum: Snac_Force (Force.c:53-188), then
// Snac_UpdateNodeMomentum_PreProcess (UpdateNode.c:74-158) and
// Snac_UpdateNodeMomentum (UpdateNode.c:60-72) for every node.  Coordinates
// are read from pos and written to pos_next, so every force sees the old
// geometry, as in the reference where all forces are summed before any node moves.
// ======================================================================================
// SnacWinklerForce (Snac/plugins/winkler/Force.c:56-168), appended to the
// force of a bottom node (j == 0): for each incident element, the isostatic
// pressure corrected by the element's bottom height acts on its bottom face
// (tets 1, 2, 6, 8, faces 0, 1, 2, 2); at step 1 the node's total y force is
// kept as a residual and subtracted from then on.
// The force-BC plugins run for a few boundary nodes only, as calls.  Their
// arguments are plain values: a reference to the kernel's parameter structs
// (or to the caller's force registers) would make every thread copy those to
// its stack before the call.
struct WinklerArgs {
    const double4* pos;
    const unsigned char* mat;
    const DevMaterial* mats;
    double* residual_fr;
    long long time_step;
    double pisos, gravity, rzbo;
};

__device__ __noinline__ V3 winkler_force(WinklerArgs a, int nx, int ny, int nz, long long n, int i, int k, V3 f) {
    Mesh m{};
    m.nx = nx;
    m.ny = ny;
    m.nz = nz;
    m.nnx = nx + 1;
    m.nny = ny + 1;
    double fx = f.x, fy = f.y, fz = f.z;
    const double factor4 = 1.0f / 4.0f;
    const double y_node = a.pos[n].y;
    const double nodeT = 0.0;  // the temperature lookup is compiled out in the reference (#if 0)
    for (int ne = 0; ne < 8; ne++) {
        const int ei = i - 1 + (ne & 1), ej = -1 + ((ne >> 1) & 1), ek = k - 1 + ((ne >> 2) & 1);
        if (ei < 0 || ej < 0 || ek < 0 || ei >= m.nx || ej >= m.ny || ek >= m.nz) continue;
        const long long e = (long long)ei + (long long)ej * m.nx + (long long)ek * m.nx * m.ny;
        const DevMaterial& M = a.mats[a.mat ? (int)a.mat[e] : 0];
        V3 corner[8];
#pragma unroll
        for (int cc = 0; cc < 8; cc++) {
            double4 p = a.pos[corner_node(m, ei, ej, ek, cc)];
            corner[cc] = {p.x, p.y, p.z};
        }
        const double phsDensity = M.density, drosub = 0.0f;
        const double p_est = a.pisos + 0.5f * (phsDensity + drosub) * a.gravity * (y_node - a.rzbo);
        const double rosubg = a.gravity * (phsDensity + drosub) * (1.0 - M.alpha * (nodeT - M.reftemp) + M.beta * p_est);
        const double dhE = factor4 * (corner[0].y + corner[1].y + corner[4].y + corner[5].y);
        const int ft[4][2] = {{1, 0}, {2, 1}, {6, 2}, {8, 2}};
        double area = 0.0f, A[4];
        V3 nr[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int t = ft[q][0], f = ft[q][1];
            tet_face(corner[tet_node(t, face_node(f, 0))], corner[tet_node(t, face_node(f, 1))],
                     corner[tet_node(t, face_node(f, 2))], A[q], nr[q]);
            area += A[q];
        }
        const double nx_ = factor4 * (nr[0].x + nr[1].x + nr[2].x + nr[3].x);
        const double ny_ = -1.0f * factor4 * (nr[0].y + nr[1].y + nr[2].y + nr[3].y);
        const double nz_ = factor4 * (nr[0].z + nr[1].z + nr[2].z + nr[3].z);
        area *= 0.5f;
        const double press_norm = a.pisos + rosubg * (a.rzbo - dhE);
        fx += factor4 * (press_norm * area * nx_);
        fy += factor4 * (press_norm * area * ny_);
        fz += factor4 * (press_norm * area * nz_);
    }
    if (a.time_step == 1) {  // restartTimestep == 0
        const double Fy = fy;
        if (Fy != 0.0) a.residual_fr[n] = Fy;
    }
    fy -= a.residual_fr[n];
    return V3{fx, fy, fz};
}

// SnacTractionBC's active branch (Snac/plugins/tractionBC/Force.c:43-268):
// on a right-wall node (i == nx), each incident element's right face (the
// triangles (1,2,6) and (1,6,5)) carries the fixed stress sxx = 1e8 Pa.
__device__ __noinline__ V3 traction_force(const double4* pos, int nx, int ny, int nz, int j, int k, V3 f) {
    Mesh m{};
    m.nx = nx;
    m.ny = ny;
    m.nz = nz;
    m.nnx = nx + 1;
    m.nny = ny + 1;
    double fx = f.x, fy = f.y, fz = f.z;
    const double factor4 = 1.0f / 4.0f;
    const double s00 = 1.0e+08, s01 = 0.0, s02 = 0.0, s10 = 0.0, s11 = 0.0, s12 = 0.0, s20 = 0.0, s21 = 0.0, s22 = 0.0;
    const int i = m.nnx - 1;
    for (int ne = 0; ne < 8; ne++) {
        const int ei = i - 1 + (ne & 1), ej = j - 1 + ((ne >> 1) & 1), ek = k - 1 + ((ne >> 2) & 1);
        if (ei < 0 || ej < 0 || ek < 0 || ei >= m.nx || ej >= m.ny || ek >= m.nz) continue;
        auto P = [&](int c) {
            const double4 p = pos[corner_node(m, ei, ej, ek, c)];
            return V3{p.x, p.y, p.z};
        };
        const V3 c1 = P(1), c2 = P(2), c5 = P(5), c6 = P(6);
        double a1, a2;
        V3 n1, n2;
        tet_face(c1, c2, c6, a1, n1);
        tet_face(c1, c6, c5, a2, n2);
        const double area = a1 + a2;
        const double nx_ = 0.5f * (n1.x + n2.x), ny_ = 0.5f * (n1.y + n2.y), nz_ = 0.5f * (n1.z + n2.z);
        fx += factor4 * area * (s00 * nx_ + s01 * ny_ + s02 * nz_);
        fy += factor4 * area * (s10 * nx_ + s11 * ny_ + s12 * nz_);
        fz += factor4 * area * (s20 * nx_ + s21 * ny_ + s22 * nz_);
    }
    return V3{fx, fy, fz};
}

// VONLY: cfg.vonly (a template argument, so that the gather loop of each
// instance is straight-line code)
// The tail of the node loop for node n with its summed force and inertial
// mass: force-BC plugins, FLAC local damping with the pre-update velocity
// (UpdateNode.c:102-104), v and x update, BC override; returns the node's
// max-BC-speed candidate.
__device__ __forceinline__ double node_update(const Mesh& m, const Fields& F, const Config& cfg, long long n, int i,
                                              int j, int k, double fx, double fy, double fz, double imass) {
    const double dt = F.sc->dt;
    if (cfg.winkler && cfg.gravity > 0.0 && j == 0) {
        const WinklerArgs a{F.pos, F.mat, F.mats, F.residual_fr, F.sc->time_step, cfg.pisos, cfg.gravity, cfg.rzbo};
        const V3 r = winkler_force(a, m.nx, m.ny, m.nz, n, i, k, V3{fx, fy, fz});
        fx = r.x;
        fy = r.y;
        fz = r.z;
    }
    if (cfg.traction && i == m.nnx - 1) {
        const V3 r = traction_force(F.pos, m.nx, m.ny, m.nz, j, k, V3{fx, fy, fz});
        fx = r.x;
        fy = r.y;
        fz = r.z;
    }
    double4 w = F.vel[n];
    const double demf = cfg.demf;
    auto sgn = [](double x) { return x < 0 ? -1.0f : x > 0 ? +1.0f : 0.0f; };
    fx -= demf * sgn(w.x) * fabs(fx);
    fy -= demf * sgn(w.y) * fabs(fy);
    fz -= demf * sgn(w.z) * fabs(fz);
    double dw[3] = {dt * fx, dt * fy, dt * fz};
    dvz_n(dw, imass, recip(imass));
    w.x += dw[0];
    w.y += dw[1];
    w.z += dw[2];
    uchar4 b = F.bc[n];
    if (b.x != 255) w.x = F.vbc_val[b.x * 3 + 0];
    if (b.y != 255) w.y = F.vbc_val[b.y * 3 + 1];
    if (b.z != 255) w.z = F.vbc_val[b.z * 3 + 2];
    double4 p = F.pos[n];
    p.x += dt * w.x;
    p.y += dt * w.y;
    p.z += dt * w.z;
    F.pos_next[n] = p;
    F.vel[n] = w;
    F.force[n] = make_double4(fx, fy, fz, imass);
    if (!(isfinite(w.x) && isfinite(w.y) && isfinite(w.z))) report(F.sc, SNAC_GPU_ENAN, n);
    return (b.x != 255 || b.y != 255 || b.z != 255) ? sqrt(w.x * w.x + w.y * w.y + w.z * w.z) : 0.0;
}

// Snac_Force (Force.c:53-188) for node n: the 8 incident hexes in
// HexaEL.c:529-573 order, 5 tets each (NodeToTetra/NodeToSurface); absent
// hexes are skipped (Force.c:92).  With cfg.vonly the fgrav row holds the
// tet volume: (g rho) V / 8 and (1/4 rho_i) V are formed here exactly as the
// element kernel forms them.
// VONLY: cfg.vonly (a template argument, so that the gather loop of each
// instance is straight-line code)
template <int DTTYPE, bool VONLY>
__device__ __forceinline__ void k_loop_nodes_body(const Mesh& m, const Fields& F, const Config& cfg, int lb) {
    long long n = (long long)lb * blockDim.x + threadIdx.x;
    bool active = n < m.nn;
    double vcand = 0.0;
    if (active) {
        int i, j, k;
        split3(n, m.nnx, m.nny, i, j, k);
        double fx = 0.0, fy = 0.0, fz = 0.0, imass = 0.0f;
        const double gr = VONLY ? cfg.gravity * cfg.m0.density : 0.0;
        const double f4r =
            VONLY ? (1.0f / 4.0f) * (DTTYPE == SNAC_DT_DYNAMIC ? F.sc->inertial_density0 : cfg.m0.density) : 0.0;
#pragma unroll
        for (int ne = 0; ne < 8; ne++) {
            int ei = i - 1 + (ne & 1), ej = j - 1 + ((ne >> 1) & 1), ek = k - 1 + ((ne >> 2) & 1);
            if (ei < 0 || ej < 0 || ek < 0 || ei >= m.nx || ej >= m.ny || ek >= m.nz) continue;
            long long e = (long long)ei + (long long)ej * m.nx + (long long)ek * m.nx * m.ny;
#pragma unroll
            for (int idx = 0; idx < 5; idx++) {
                const int t = node_tet(ne, idx);
                const int f = node_face(ne, idx);
                const long long R = m.ner;
                const double* o = F.fterm + (t * 12 + f * 3) * R + e;
                if (DTTYPE != SNAC_DT_CONSTANT && VONLY) {
                    const double V = F.fgrav[t * R + e];
                    imass += f4r * V;
                    fx += o[0];
                    fy += o[R];
                    fz += o[2 * R];
                    fy -= gr * V * 0.125;
                } else {
                    imass += (DTTYPE == SNAC_DT_CONSTANT) ? F.fmass[(t * 4 + f) * R + e] : F.fmass[t * R + e];
                    fx += o[0];
                    fy += o[R];
                    fz += o[2 * R];
                    fy -= F.fgrav[t * R + e];
                }
            }
        }
        vcand = node_update(m, F, cfg, n, i, j, k, fx, fy, fz, imass);
    }
    // max |v| over velocity-BC nodes for Sync (exact: max does not round)
    for (int o = 16; o > 0; o >>= 1) vcand = fmax(vcand, __shfl_xor_sync(FULL, vcand, o));
    if ((threadIdx.x & 31) == 0 && vcand > 0.0)
        atomicMax(&F.sc->vmax_bits, (unsigned long long)__double_as_longlong(vcand));
}

#ifndef SNAC_NODE_MINB
#define SNAC_NODE_MINB 8  // resident 128-thread blocks per SM asked of the node gather (64 registers; measured best)
#endif
template <int DTTYPE, bool VONLY>
__global__ void __launch_bounds__(128, SNAC_NODE_MINB) k_loop_nodes(Mesh m, Fields F, Config cfg) {
    k_loop_nodes_body<DTTYPE, VONLY>(m, F, cfg, blockIdx.x);
}

// Slab launches of the step with the state in host memory: the same bodies
// over blocks [b0, b0 + gridDim.x) of the whole-mesh launch, so a slab's
// hexes (nodes) get exactly the arithmetic of the whole-mesh kernels.
template <int PLUGIN, bool ONE>
__global__ void __launch_bounds__(ELEM_WARPS * 32, SNAC_ELEM_MINB) k_calc_stresses_slab(Mesh m, Fields F, Config cfg,
                                                                                        int b0) {
    k_calc_stresses_body<PLUGIN, ONE>(m, F, cfg, b0 + (int)blockIdx.x);
}

// UpdateElement.c:54-269 with this step's dt and the minimum length scale
// of the new geometry (the unfused element update)
template <int PLUGIN>
__global__ void __launch_bounds__(ELEM_WARPS * 32, SNAC_ELEM_MINB) k_update_elements_slab(Mesh m, Fields F, Config cfg,
                                                                                          int b0) {
    k_update_elements_body<PLUGIN>(m, F, cfg, 0, b0 + (int)blockIdx.x);
}

template <int DTTYPE, bool VONLY>
__global__ void __launch_bounds__(128, SNAC_NODE_MINB) k_loop_nodes_slab(Mesh m, Fields F, Config cfg, int b0) {
    k_loop_nodes_body<DTTYPE, VONLY>(m, F, cfg, b0 + (int)blockIdx.x);
}

// ======================================================================================
// Snac_EP_LoopElementsEnergy: Snac_HeatFlux (temperature/HeatFlux.c:60-200) and
// SnacTemperature_HeatFluxBC (temperature/VariableConditions.c:280-413)
// ======================================================================================
template <bool ONE>
__device__ __forceinline__ void heat_flux_tet(const Mesh& m, const Fields& F, const Config& cfg, const TetSlot& s,
                                              const double T[4], const double T0[4], const TetGeom& g) {
    const DevMaterial& M = ONE ? cfg.m0 : F.mats[s.active ? phase_of(F, s.e) : 0];
    double q[3], tsr = 0.0;
    const double zV = g.zV;
#pragma unroll
    for (int d = 0; d < 3; d++)
        q[d] = 1.0f * M.thermal_conduct *
               (T[0] * comp(g.n[1], d) * g.A[1] + T[1] * comp(g.n[2], d) * g.A[2] + T[2] * comp(g.n[3], d) * g.A[3] +
                T[3] * comp(g.n[0], d) * g.A[0]);
    dvk_n(q, 3.0, Z3);
    dvz_n(q, g.V, zV);
    if (cfg.thermal_stress) {
        const double bulkm = M.lambda + dv3(2.0f * M.mu);
        double temp = 0.25f * (T[0] + T[1] + T[2] + T[3]);
        double temp0 = 0.25f * (T0[0] + T0[1] + T0[2] + T0[3]);
        tsr = -1.0f * M.alpha * bulkm * (temp - temp0);
    }
    // flux BC on the x and z walls: remove the wall-normal part of grad T
    const bool on_wall = s.active && (s.i == 0 || s.i == m.nx - 1 || s.k == 0 || s.k == m.nz - 1);
    double nrm[4][3];
    // (tet, face) pairs averaged for each wall, VariableConditions.c:311-367;
    // the shuffles run only in warps that hold a wall element (warp-uniform)
    if (__any_sync(FULL, on_wall)) {
        const int W[4][4][2] = {{{0, 2}, {1, 2}, {5, 0}, {6, 0}},
                                {{2, 0}, {3, 0}, {7, 0}, {8, 0}},
                                {{0, 1}, {2, 2}, {6, 1}, {7, 1}},
                                {{1, 1}, {3, 2}, {5, 1}, {8, 1}}};
#pragma unroll
        for (int w = 0; w < 4; w++)
#pragma unroll
            for (int d = 0; d < 3; d++) {
                double a[4];
#pragma unroll
                for (int r = 0; r < 4; r++) {
                    const int f = W[w][r][1];
                    double val = f == 0 ? comp(g.n[0], d) : f == 1 ? comp(g.n[1], d) : f == 2 ? comp(g.n[2], d) : comp(g.n[3], d);
                    a[r] = __shfl_sync(FULL, val, s.base + W[w][r][0]);
                }
                nrm[w][d] = 0.25f * (a[0] + a[1] + a[2] + a[3]);
            }
    }
    if (on_wall) {
        double normal[3];
        if (s.i == 0)
            for (int d = 0; d < 3; d++) normal[d] = nrm[0][d];
        if (s.i == m.nx - 1)
            for (int d = 0; d < 3; d++) normal[d] = nrm[1][d];
        if (s.k == 0)
            for (int d = 0; d < 3; d++) normal[d] = nrm[2][d];
        if (s.k == m.nz - 1)
            for (int d = 0; d < 3; d++) normal[d] = nrm[3][d];
        double gd[3];
        for (int d = 0; d < 3; d++)
            gd[d] = dvz(dv3(-1.0f * (T[0] * comp(g.n[1], d) * g.A[1] + T[1] * comp(g.n[2], d) * g.A[2] +
                                     T[2] * comp(g.n[3], d) * g.A[3] + T[3] * comp(g.n[0], d) * g.A[0])),
                        g.V, zV);
        double Fn = 0.0f;
        for (int d = 0; d < 3; d++) Fn += gd[d] * normal[d];
        for (int d = 0; d < 3; d++) q[d] -= Fn * normal[d];
    }
    // Per-tet terms of Snac_Heat (temperature/Heat.c:88-126) for the node
    // gather: (q . n) A / 6 of each face, the lumped heat capacity
    // Cp rho V / 8, and the thermal stress for the visco-plastic hook.
    if (s.active) {
        const long long R = m.ner;
        double* h = F.hflux + (long long)(s.t * HF_STRIDE) * R + s.e;
        double hf[4];
#pragma unroll
        for (int f = 0; f < 4; f++) hf[f] = (q[0] * g.n[f].x + q[1] * g.n[f].y + q[2] * g.n[f].z) * g.A[f];
        dvk_n(hf, 6.0, Z6);
#pragma unroll
        for (int f = 0; f < 4; f++) h[f * R] = hf[f];
        // tetra density is set from TimeStepZero on, so the reference's
        // "density == 0" fallback (Heat.c:120-125) is never taken
        const double rho = cfg.has_density ? F.density[s.q] : M.density;
        h[4 * R] = M.heat_capacity * ((rho)*g.V) * 0.125;  // rounds as / 8
        if (cfg.thermal_stress) h[5 * R] = tsr;
        // Heat.c:127-135, once per element; with one phase every element
        // gives the same value, so only element 0 (the first the reference
        // checks) evaluates it
        if (s.t == 0 && (!ONE || s.e == 0)) {
            double dt_thermal_to_mech = sqrt((M.lambda + 2.0f * M.mu) / M.density) * F.sc->min_length_scale /
                                        (M.thermal_conduct / (M.heat_capacity * M.density));
            if (!(dt_thermal_to_mech > 1.0)) report(F.sc, SNAC_GPU_EPHYSICS, s.e);
        }
    }
}

template <bool ONE>
__device__ __forceinline__ void k_heat_flux_body(const Mesh& m, const Fields& F, const Config& cfg, int lb) {
    TetSlot s = tet_slot(m, lb);
    V3 c[4], v[4];
    double T[4], T0[4];
    load_tet(m, F, s, c, v, T, T0);
    TetGeom g;
    tet_geometry(c, g);
    heat_flux_tet<ONE>(m, F, cfg, s, T, T0, g);
}

#ifndef SNAC_HEAT_MINB
#define SNAC_HEAT_MINB 6  // resident blocks per SM asked of the heat-flux kernel (80 registers; measured best)
#endif
template <bool ONE>
__global__ void __launch_bounds__(ELEM_WARPS * 32, SNAC_HEAT_MINB) k_heat_flux(Mesh m, Fields F, Config cfg,
                                                                           int count_step) {
    if (count_step && blockIdx.x == 0 && threadIdx.x == 0) {  // the step's first kernel: timeStep++, currentTime += dt
        F.sc->time_step += 1;
        F.sc->current_time += F.sc->dt;
    }
    k_heat_flux_body<ONE>(m, F, cfg, blockIdx.x);
}


// ======================================================================================
// Snac_EP_LoopNodesEnergy: Snac_Heat for every node (temperature/Heat.c:64-140),
// the tet mean temperatures and the temperature BCs (Heat.c:47-62)
// ======================================================================================
__device__ __forceinline__ void k_heat_nodes_body(const Mesh& m, const Fields& F, const Config& cfg, int lb) {
    long long n = (long long)lb * blockDim.x + threadIdx.x;
    if (n >= m.nn) return;
    const double dt = F.sc->dt;
    int i, j, k;
    split3(n, m.nnx, m.nny, i, j, k);
    double energy = 0.0f, lumpVolume = 0.0f;
    // the volumetric source of Snac_Heat is called with sourceterm = 0
    // (Heat.c:59), which adds +0 to the energy
    const double source = 0.0f;
#pragma unroll
    for (int ne = 0; ne < 8; ne++) {
        int ei = i - 1 + (ne & 1), ej = j - 1 + ((ne >> 1) & 1), ek = k - 1 + ((ne >> 2) & 1);
        if (ei < 0 || ej < 0 || ek < 0 || ei >= m.nx || ej >= m.ny || ek >= m.nz) continue;
        long long e = (long long)ei + (long long)ej * m.nx + (long long)ek * m.nx * m.ny;
#pragma unroll
        for (int idx = 0; idx < 5; idx++) {
            const long long R = m.ner;
            const double* h = F.hflux + (node_tet(ne, idx) * HF_STRIDE) * R + e;
            energy += h[node_face(ne, idx) * R];
            lumpVolume += h[4 * R];
        }
    }
    // only the w slots are written: other threads read this node's x, y, z
    double* pw = reinterpret_cast<double*>(const_cast<double4*>(F.pos) + n) + 3;
    double Told = *pw;
    double Tnew = Told + dv((energy + source) * -1.0f * dt, lumpVolume);
    if (F.tpre) F.tpre[n] = Tnew;
    uchar4 b = F.bc[n];
    if (b.w != 255) Tnew = F.tbc_val[b.w];
    reinterpret_cast<double*>(F.vel + n)[3] = Told;
    *pw = Tnew;
    if (!isfinite(Tnew)) report(F.sc, SNAC_GPU_ENAN, n);
}

// count_step: the step's first kernel (its heat flux was formed at the end
// of the previous step): timeStep++, currentTime += dt
__global__ void __launch_bounds__(128) k_heat_nodes(Mesh m, Fields F, Config cfg, int count_step) {
    if (count_step && blockIdx.x == 0 && threadIdx.x == 0) {
        F.sc->time_step += 1;
        F.sc->current_time += F.sc->dt;
    }
    k_heat_nodes_body(m, F, cfg, blockIdx.x);
}

// Slab launches of the energy hooks for the step with the state in host
// memory (see k_calc_stresses_slab): blocks [b0, b0 + gridDim.x) of the
// whole-mesh launch; the step was counted by its first kernel.
template <bool ONE>
__global__ void __launch_bounds__(ELEM_WARPS * 32, SNAC_HEAT_MINB) k_heat_flux_slab(Mesh m, Fields F, Config cfg,
                                                                                   int b0) {
    k_heat_flux_body<ONE>(m, F, cfg, b0 + (int)blockIdx.x);
}

__global__ void __launch_bounds__(128) k_heat_nodes_slab(Mesh m, Fields F, Config cfg, int b0) {
    k_heat_nodes_body(m, F, cfg, b0 + (int)blockIdx.x);
}

// ======================================================================================
// AbstractContext_EP_Sync: _Snac_Context_Sync (Context.c:1208-1268), one thread
// ======================================================================================
__device__ __forceinline__ void sync_one(const Config& cfg, DevScalars* sc, double wave_speed) {
    // the reductions are read where the other blocks' atomics left them (L2)
    double vmax = __longlong_as_double((long long)atomicOr(&sc->vmax_bits, 0ull));
    const double vlb = 3.0e-11f;
    if (vmax < vlb) vmax = vlb;
    sc->vmax = vmax;
    double minLS = __longlong_as_double((long long)atomicOr(&sc->minls_bits, 0ull));
    sc->min_length_scale = minLS;
    if (sc->time_step == 0) sc->init_min_length_scale = minLS;
    sc->dt_rot = sc->dt;  // the element update of this step (done now, or deferred into the next kernel) used this dt
    if (cfg.dt_type == SNAC_DT_DYNAMIC) {
        sc->dt = minLS * 0.45f * cfg.strain_inert / vmax;
        sc->speed_of_sound = minLS * 0.5f / sc->dt;
        // Force.c:112-114 for phase 0, once per step instead of once per tet
        sc->inertial_density0 = dv(cfg.m0.lambda + 2.0f * cfg.m0.mu, sc->speed_of_sound * sc->speed_of_sound);
    } else if (cfg.dt_type == SNAC_DT_WAVE) {
        sc->speed_of_sound = wave_speed;
        sc->dt = 0.5f * minLS / sc->speed_of_sound;
    }
    sc->vmax_bits = 0ull;
    sc->minls_bits = 0x7ff0000000000000ull;  // +inf
}

// The minimum length scale of the new coordinates and Sync in one launch:
// the last block to finish (counted in DevScalars, reset by that block) runs
// Sync on the completed reductions.
constexpr int MINLS_THREADS = 128;  // one thread per hex
__global__ void __launch_bounds__(MINLS_THREADS) k_min_length_scale_sync(Mesh m, Fields F, Config cfg,
                                                                         double wave_speed) {
    double ls = hex_min_length_scale(m, F, blockIdx.x);
    for (int o = 16; o > 0; o >>= 1) ls = fmin(ls, __shfl_xor_sync(FULL, ls, o));
    // the block's minimum in one atomic (fewer atomics on the one address),
    // fenced so that it is visible device-wide before the block is counted
    __shared__ double wmin[MINLS_THREADS / 32];
    __shared__ bool last;
    if ((threadIdx.x & 31) == 0) wmin[threadIdx.x >> 5] = ls;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = wmin[0];
#pragma unroll
        for (int w = 1; w < MINLS_THREADS / 32; w++) b = fmin(b, wmin[w]);
        atomicMin(&F.sc->minls_bits, (unsigned long long)__double_as_longlong(b));
        __threadfence();
        last = atomicAdd(&F.sc->blocks_done, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        sync_one(cfg, F.sc, wave_speed);
        F.sc->blocks_done = 0u;
    }
}

// Temperature runs: the minimum length scale of step n together with the
// heat flux of step n+1 (Snac_HeatFlux, temperature/HeatFlux.c:60-200, and
// its wall BC), which reads the same coordinates x^{n+1} and node
// temperatures T^{n+1}: one geometry evaluation instead of two.  One thread
// per tet, as k_heat_flux; each block's minimum goes to one of 32 slots
// (non-returning atomics spread over addresses, so that the many small
// blocks neither queue on one address nor wait for a counter), and
// k_slots_sync then takes the minimum of the slots and runs Sync.  The tet's
// share of the minimum is RN(V / max_f A_f) from the heat flux's own face areas:
// max_f RN(RN(sqrt(s_f)) / 2) = RN(RN(sqrt(max_f s_f)) / 2), square root and
// halving being monotonic and correctly rounded (faces with a NaN area are
// skipped by both forms), so the minimum has the bits of
// hex_min_length_scale.
#ifndef SNAC_HEAT_MINLS_MINB
#define SNAC_HEAT_MINLS_MINB 5  // resident blocks per SM asked of the kernel below
#endif
template <bool ONE>
__global__ void __launch_bounds__(ELEM_WARPS * 32, SNAC_HEAT_MINLS_MINB)
    k_heat_flux_min_length_scale(Mesh m, Fields F, Config cfg) {
    TetSlot s = tet_slot(m, blockIdx.x);
    V3 c[4], v[4];
    double T[4], T0[4];
    load_tet(m, F, s, c, v, T, T0);
    TetGeom g;
    tet_geometry(c, g);
    heat_flux_tet<ONE>(m, F, cfg, s, T, T0, g);
    double ls = 1.0e+27f;
    if (s.active) {
        double A = 0.0;
#pragma unroll
        for (int f = 0; f < 4; f++)
            if (g.A[f] > A) A = g.A[f];
        if (A) {
            const double l = fabs(dv(g.V, A));
            if (ls > l) ls = l;
        }
        if (g.V == 0.0) report(F.sc, SNAC_GPU_EVOLUME, s.e);
    }
    for (int o = 16; o > 0; o >>= 1) ls = fmin(ls, __shfl_xor_sync(FULL, ls, o));
    __shared__ double wmin[ELEM_WARPS];
    if ((threadIdx.x & 31) == 0) wmin[threadIdx.x >> 5] = ls;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = wmin[0];
#pragma unroll
        for (int w = 1; w < ELEM_WARPS; w++) b = fmin(b, wmin[w]);
        atomicMin(&F.sc->minls_slot[blockIdx.x & 31], (unsigned long long)__double_as_longlong(b));
    }
}

// One warp after k_heat_flux_min_length_scale: the minimum over its
// slots (exact: min does not round), the slots reset, then Sync.
__global__ void k_slots_sync(Config cfg, DevScalars* sc, double wave_speed) {
    const int l = threadIdx.x;
    unsigned long long v = sc->minls_slot[l];
    sc->minls_slot[l] = 0x7ff0000000000000ull;
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long w = __shfl_xor_sync(FULL, v, o);
        v = w < v ? w : v;
    }
    if (l == 0) {
        if (v < sc->minls_bits) sc->minls_bits = v;
        sync_one(cfg, sc, wave_speed);
    }
}

__global__ void k_sync(Config cfg, DevScalars* sc, double wave_speed) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    sync_one(cfg, sc, wave_speed);
}

// max |v| over the velocity-BC nodes from the current velocities, for a
// Sync that does not follow the node loop (step zero, hook-by-hook callers)
__device__ __forceinline__ void k_vmax_body(const Mesh& m, const Fields& F, int lb) {
    long long n = (long long)lb * blockDim.x + threadIdx.x;
    double vcand = 0.0;
    if (n < m.nn) {
        uchar4 b = F.bc[n];
        if (b.x != 255 || b.y != 255 || b.z != 255) {
            double4 w = F.vel[n];
            vcand = sqrt(w.x * w.x + w.y * w.y + w.z * w.z);
        }
    }
    for (int o = 16; o > 0; o >>= 1) vcand = fmax(vcand, __shfl_xor_sync(FULL, vcand, o));
    if ((threadIdx.x & 31) == 0 && vcand > 0.0)
        atomicMax(&F.sc->vmax_bits, (unsigned long long)__double_as_longlong(vcand));
}

__global__ void __launch_bounds__(256) k_vmax(Mesh m, Fields F) {
    k_vmax_body(m, F, blockIdx.x);
}

// ======================================================================================
// Surface-topography diffusion (UpdateNode.c:161-857, cartesian), after the node update.
// The reference runs getMaxTopoGrad, DiffTopo + UpdateInteriorTopo and
// AdjustEdgeTopo inside its node loop, node after node: a top node sees its
// -x and -z neighbours already finished (moved, diffused, edge-copied) and
// its +x and +z neighbours not yet moved this step (their start-of-step
// coordinates).  That is a wavefront over the top surface's anti-diagonals
// i + k = d: one block walks the diagonals in order, the nodes of a diagonal
// in parallel.  topoGradMax is the running max in node order (a prefix max,
// exact in any association), never reset between steps.
// old: start-of-step coordinates; cur: after this step's node update (updated in place).
// tgrad: scratch of (nnx * nnz) doubles.
// ======================================================================================
__global__ void __launch_bounds__(1024) k_topo(Mesh m, const double4* __restrict__ old, double4* cur, Config cfg,
                                               DevScalars* sc, double* tgrad) {
    __shared__ double chunk_max[1024];
    if (sc->time_step <= 1) return;
    const int nnx = m.nnx, nnz = m.nnz, T = blockDim.x, tid = threadIdx.x;
    const long long top = (long long)(m.nny - 1) * nnx, plane = (long long)nnx * m.nny;
    const long long N = (long long)nnx * nnz;
    auto id = [&](int i, int k) { return (long long)i + top + (long long)k * plane; };
    auto interior = [&](int i, int k) { return i > 0 && i < nnx - 1 && k > 0 && k < nnz - 1; };
    // getMaxTopoGrad (:161-260), called from UpdateNodeMomentum when topo_kappa > 0
    for (long long p = tid; p < N; p += T) {
        const int i = (int)(p % nnx), k = (int)(p / nnx);
        double g = -CUDART_INF;
        if (cfg.topo_kappa > 0 && interior(i, k)) {
            const double4 X0 = cur[id(i, k)], xR = old[id(i + 1, k)], xF = old[id(i, k + 1)];
            const double dydx = (xR.y - X0.y) / (xR.x - X0.x);
            const double dydz = (xF.y - X0.y) / (xF.z - X0.z);
            g = sqrt(dydx * dydx + dydz * dydz);
        }
        tgrad[p] = g;
    }
    __syncthreads();
    // running max in node order: each thread a contiguous chunk, then the chunk prefixes
    const long long C = (N + T - 1) / T, lo = tid * C, hi = lo + C < N ? lo + C : N;
    double cm = -CUDART_INF;
    for (long long p = lo; p < hi; p++) cm = cm > tgrad[p] ? cm : tgrad[p];
    chunk_max[tid] = cm;
    __syncthreads();
    if (tid == 0) {
        double run = sc->topo_grad_max;
        for (int t = 0; t < T; t++) {
            const double c = chunk_max[t];
            chunk_max[t] = run;  // the max before chunk t
            run = run > c ? run : c;
        }
        sc->topo_grad_max = run;
    }
    __syncthreads();
    double run = chunk_max[tid];
    for (long long p = lo; p < hi; p++) {
        run = run > tgrad[p] ? run : tgrad[p];
        tgrad[p] = run;  // topoGradMax as node p's DiffTopo sees it
    }
    __syncthreads();
    const double kdt = cfg.topo_kappa * sc->dt;
    for (int d = 0; d <= (nnx - 1) + (nnz - 1); d++) {
        const int i0 = d - (nnz - 1) > 0 ? d - (nnz - 1) : 0, i1 = d < nnx - 1 ? d : nnx - 1;
        for (int i = i0 + tid; i <= i1; i += T) {
            const int k = d - i;
            if (tgrad[i + (long long)k * nnx] < cfg.topo_crit) continue;  // "topoGradMax < topoGradCriterion"
            double4& X0 = cur[id(i, k)];
            if (interior(i, k)) {
                // DiffTopo (:359-506) and UpdateInteriorTopo (:647-715)
                const double4 xR = old[id(i + 1, k)], xF = old[id(i, k + 1)];
                const double4 xL = cur[id(i - 1, k)], xB = cur[id(i, k - 1)];
                const double dydx1 = (xR.y - X0.y) / (xR.x - X0.x);
                const double dydx2 = (X0.y - xL.y) / (X0.x - xL.x);
                const double d2ydx2 = (dydx1 - dydx2) / (0.5f * (xR.x - xL.x));
                const double dydz1 = (xF.y - X0.y) / (xF.z - X0.z);
                const double dydz2 = (X0.y - xB.y) / (X0.z - xB.z);
                const double d2ydz2 = (dydz1 - dydz2) / (0.5f * (xF.z - xB.z));
                const double lapl_topo = d2ydx2 + d2ydz2;
                X0.y += kdt * lapl_topo;
            } else {
                // AdjustEdgeTopo (:716-857): copy the neighbour's height inward
                bool h1 = false, h2 = false;
                double y1 = 0.0, y2 = 0.0;
                if (i == 0) {
                    h1 = true;
                    y1 = old[id(1, k)].y;
                } else if (i == nnx - 1) {
                    h1 = true;
                    y1 = cur[id(nnx - 2, k)].y;
                }
                if (k == 0) {
                    h2 = true;
                    y2 = old[id(i, 1)].y;
                } else if (k == nnz - 1) {
                    h2 = true;
                    y2 = cur[id(i, nnz - 2)].y;
                }
                if (h1 && !h2) X0.y = y1;
                else if (!h1 && h2) X0.y = y2;
                else if (h1 && h2) X0.y = 0.5f * (y1 + y2);
            }
        }
        __syncthreads();
    }
}

// ---- self-test of the straight-line division against the IEEE quotient -------------------
__device__ __forceinline__ unsigned long long splitmix64(unsigned long long& x) {
    unsigned long long z = (x += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
__device__ __forceinline__ bool same_bits(double a, double b) {
    return __double_as_longlong(a) == __double_as_longlong(b) || (a != a && b != b);
}
__global__ void k_selftest_division(long long n, unsigned long long seed, unsigned long long* bad) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long st = seed ^ (0x632be59bd9b4e019ull * (unsigned long long)(i + 1));
    unsigned long long local = 0;
    for (; i < n; i += (long long)gridDim.x * blockDim.x) {
        unsigned long long a = splitmix64(st), b = splitmix64(st), c = splitmix64(st);
        // random significands, exponents spread over +-300 (x) and +-130 (y), random signs
        double x = __longlong_as_double((long long)((a & 0x800fffffffffffffull) | ((unsigned long long)(1023 + (int)(c % 601) - 300) << 52)));
        double y = __longlong_as_double((long long)((b & 0x800fffffffffffffull) | ((unsigned long long)(1023 + (int)((c >> 20) % 261) - 130) << 52)));
        if ((c >> 40) % 5 == 0) x = rint(x * 1e-3) * y;         // quotients that are exact or near ties
        if ((c >> 44) % 97 == 0) x = ((c >> 50) & 1) ? 0.0 : -0.0;
        // about 1 in 16: an operand drawn from every exponent (subnormals,
        // zeros' neighbours, overflow range, Inf and NaN) to exercise the window tests
        unsigned long long d = splitmix64(st);
        if ((d & 15) == 0) x = __longlong_as_double((long long)((a & 0x800fffffffffffffull) | ((d >> 8) % 2048) << 52));
        if (((d >> 4) & 15) == 0) y = __longlong_as_double((long long)((b & 0x800fffffffffffffull) | ((d >> 20) % 2048) << 52));
        local += !same_bits(dv(x, y), x / y);
        local += !same_bits(dvz(x, y, recip(y)), x / y);
        local += !same_bits(dv3(x), x / 3.0) + !same_bits(dv6(x), x / 6.0);
        local += !same_bits(dv9(x), x / 9.0) + !same_bits(dv10(x), x / 10.0);
    }
    if (local) atomicAdd(bad, local);
}

// ---- host transfers: node fields between the packed double4 layout and
// the reference's interleaved (x, y, z) / scalar arrays -------------------------------------
// what: 0 = x, y, z of each double4 <-> 3 doubles per node; 1 = w <-> 1 double per node
__global__ void k_pack_nodes(const double4* __restrict__ src, double* __restrict__ dst, long long nn, int what) {
    long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nn) return;
    double4 a = src[n];
    if (what == 0) {
        dst[n * 3 + 0] = a.x;
        dst[n * 3 + 1] = a.y;
        dst[n * 3 + 2] = a.z;
    } else {
        dst[n] = a.w;
    }
}

__global__ void k_unpack_nodes(double4* __restrict__ dst, const double* __restrict__ src, long long nn, int what) {
    long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nn) return;
    double* d = reinterpret_cast<double*>(dst + n);
    if (what == 0) {
        d[0] = src[n * 3 + 0];
        d[1] = src[n * 3 + 1];
        d[2] = src[n * 3 + 2];
    } else {
        d[3] = src[n];
    }
}

// The node state of nodes [0, nn) between the host's rows (3 doubles of
// coordinates, 3 of velocity, 1 of temperature per node) and the device's
// double4 rows (pos: x, y, z, T; vel: vx, vy, vz and the previous T, which
// stays); pos and vel always hold nn rows, a null host row (c, t, v) is
// skipped.
__global__ void k_unpack_node_state(double4* __restrict__ pos, const double* __restrict__ c,
                                    const double* __restrict__ t, double4* __restrict__ vel,
                                    const double* __restrict__ v, long long nn) {
    long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nn) return;
    double* p = reinterpret_cast<double*>(pos + n);
    if (c) {
        p[0] = c[n * 3 + 0];
        p[1] = c[n * 3 + 1];
        p[2] = c[n * 3 + 2];
    }
    if (t) p[3] = t[n];
    if (v) {
        double* w = reinterpret_cast<double*>(vel + n);
        w[0] = v[n * 3 + 0];
        w[1] = v[n * 3 + 1];
        w[2] = v[n * 3 + 2];
    }
}

__global__ void k_pack_node_state(const double4* __restrict__ pos, double* __restrict__ c, double* __restrict__ t,
                                  const double4* __restrict__ vel, double* __restrict__ v, long long nn) {
    long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nn) return;
    const double4 x = pos[n];
    if (c) {
        c[n * 3 + 0] = x.x;
        c[n * 3 + 1] = x.y;
        c[n * 3 + 2] = x.z;
    }
    if (t) t[n] = x.w;
    if (v) {
        const double4 w = vel[n];
        v[n * 3 + 0] = w.x;
        v[n * 3 + 1] = w.y;
        v[n * 3 + 2] = w.z;
    }
}

// _AbstractContext_Execute_Hook: timeStep++ and dt = dtFactor * dt (AbstractContext.c:874-890)
__global__ void k_begin_step(DevScalars* sc) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        sc->time_step += 1;
        sc->dt = 1.0 * sc->dt;
        sc->current_time += sc->dt;
    }
}

}  // namespace snac
