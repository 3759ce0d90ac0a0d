// snac_adjoint.cuh — hand-written reverse mode of the SNAC step (FP64).
//
// Gradients of a loss on the final top-surface vertical velocity and
// topography with respect to the per-element cohesion, friction-angle and
// viscosity scales (Fields::coh_scale / fric_scale / visc_scale) and to the
// entry state (coordinates, velocities, tet stresses, plastic strains), for
// the elastic, Maxwell, Mohr-Coulomb plastic and visco-plastic constitutive
// hooks with a constant dt.  The temperature field is held fixed (zero
// conductivity).
//
// Forward step n (what is differentiated; the per-tet operations are those
// of csrc/snac_kernels.cuh):
//   sigma_pre^n = Rot(sigma_avg^{n-1}, v^n, G(x^n))       (end of step n-1)
//   sr          = StrainRate(v^n, G(x^n)) + mixed averaging over the hex
//   sigma_c     = Constitutive(sigma_pre^n, sr dt, eps_p^n, scales)
//                 (Maxwell: also the volume ratio V(x^n) / V(x^{n-1}))
//   sigma_avg^n = trace averaging of sigma_c over the hex
//   F, m        = Force(sigma_avg^n, G(x^n))                (node gather)
//   v^{n+1}     = v^n + dt damp(F, v^n) / m   (BC components fixed)
//   x^{n+1}     = x^n + dt v^{n+1}
// The reverse of step n is split in two kernels: k_adj_tet (one thread per
// tet: forward recompute of the tet from the stored state, then the reverse
// of Force, averaging, Constitutive, StrainRate, Rot of step n-1 and the
// geometry) and k_adj_nodes (one thread per node: gather of the per-tet
// corner adjoints in a fixed order, then the reverse of the node update of
// the previous step).  No atomics: the gradients are bit-reproducible.
//
// The return map is differentiated along the branch the forward took
// (elastic / shear / tension), through the eigen-decomposition of the trial
// stress (the Daleckii-Krein form of the derivative of a spectral function).
// sgn() in the FLAC damping and the viscosity clip are differentiated as the
// piecewise-constant functions they are.
#pragma once

#include "snac_kernels.cuh"

namespace snac {

// one stored forward state between steps (the fused pipeline's state: the
// stress of step n-1 still to be rotated, except at n = 0)
struct AdjState {
    const double4* pos;    // x^n (w: temperature)
    const double4* vel;    // v^n
    const double4* force;  // damped force and inertial mass of step n-1
    const double* stress;  // sigma_avg^{n-1} (n >= 1) or sigma_pre^0 (n = 0)
    const double* eps_p;   // eps_p^n
    const double* vol;     // [nq][2] Maxwell: tet volume and old volume as stored (else null)
};

struct AdjBufs {
    double4* xbar;   // [nn] adjoint of x (w unused)
    double4* vbar;   // [nn] adjoint of v
    double4* fbar;   // [nn] adjoint of the damped-force input F (xyz) and of the inertial mass (w)
    double* cbuf;    // per-tet corner adjoints (x 3, v 3) for the node gather: rows (t, corner, component) of ner hexes
    double* sbar;    // [nq][6] adjoint of sigma_avg^{n-1}, handed to the next (earlier) step
    double* epbar;   // [nq] adjoint of eps_p
    double* pbar;    // [nq][3] adjoint of the cohesion, friction, viscosity scales
    double* vobar;   // [nq] Maxwell: adjoint of the volume pass n stored, handed to pass n-1
};

struct D3 {
    double x, y, z;
};
__device__ __forceinline__ D3 d3(double x, double y, double z) { return {x, y, z}; }
__device__ __forceinline__ D3 operator-(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ D3 operator+(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ D3 operator*(double s, D3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ D3 cross(D3 a, D3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
__device__ __forceinline__ double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ double cmp(const D3& a, int d) { return d == 0 ? a.x : (d == 1 ? a.y : a.z); }
__device__ __forceinline__ void addc(D3& a, int d, double v) {
    if (d == 0) a.x += v;
    else if (d == 1) a.y += v;
    else a.z += v;
}
__device__ __forceinline__ double sgnd(double x) { return x < 0 ? -1.0 : (x > 0 ? 1.0 : 0.0); }

#ifndef SNAC_ADJ_SMEM_REC
#define SNAC_ADJ_SMEM_REC 1  // the forward record in shared memory (fewer spills; measured faster)
#endif
// ---- forward record of the constitutive update of one tet --------------------------------
struct ConsRec {
    // visco-plastic Maxwell step
    double trs, tre, d[3], sd[3], Q, J, eta, eta_base, vic1, vic2, tmp;
    bool J_from_sqrt, eta_free;
    // Maxwell hook: whether the tet's phase takes the update, and the volume
    // ratio its trace strain is formed from
    bool mx;
    double vcur, vold;
    // softening lookup
    double co, hd, fa, da, fa_b, co_b, dpl, tgf_b, tgc_b, tgd;
    bool clamped;
    double sphi, spsi, anphi, anpsi, stc;
    bool stc_from_co;
    // return map
    bool yield, tension;
    double sp[3], sq[3], cn[3][3], alam, inc;
};

// ---- reverse of the MC return map (spectral part + principal-space update) ------------------
// in: sbar_out (6, adjoint of the stress after the map), epbar_out (adjoint
// of eps_p after the map).  out: sbar_in (6), and adjoints of the softening
// quantities (co, hd, anphi, anpsi, stc), plus epbar accumulated.
__device__ __forceinline__ void mc_reverse(const ConsRec& R, const double sb_out[6], double epb_out, double a1,
                                           double a2, double sb_in[6], double& cob, double& hdb, double& anphib,
                                           double& anpsib, double& stcb) {
    // B = C^T Mbar C with Mbar the symmetric matrix of the 6-vector adjoint
    double Mb[3][3] = {{sb_out[0], 0.5 * sb_out[3], 0.5 * sb_out[4]},
                       {0.5 * sb_out[3], sb_out[1], 0.5 * sb_out[5]},
                       {0.5 * sb_out[4], 0.5 * sb_out[5], sb_out[2]}};
    double B[3][3];
    for (int k = 0; k < 3; k++)
        for (int l = 0; l < 3; l++) {
            double acc = 0.0;
            for (int a = 0; a < 3; a++)
                for (int b = 0; b < 3; b++) acc += R.cn[k][a] * Mb[a][b] * R.cn[l][b];
            B[k][l] = acc;
        }
    // principal-space update sq = g(sp)
    double spb[3] = {B[0][0], B[1][1], B[2][2]};  // adjoint of sq, becomes adjoint of sp
    const double sqan = sqrt(R.anphi);
    double alamb = 0.0;
    // plastic strain increment inc = sqrt(h(dep)), dep = alam * (1, 0, -anpsi) or (0, 0, 1)
    double dep[3];
    if (!R.tension) {
        dep[0] = R.alam;
        dep[1] = 0.0;
        dep[2] = -R.alam * R.anpsi;
    } else {
        dep[0] = 0.0;
        dep[1] = 0.0;
        dep[2] = R.alam;
    }
    const double depm = (dep[0] + dep[1] + dep[2]) / 3.0;
    double depb[3] = {0, 0, 0};
    if (R.inc > 0.0) {
        const double hb = epb_out / (2.0 * R.inc);
        for (int i = 0; i < 3; i++) depb[i] = hb * ((dep[i] - depm) + depm / 3.0);
    }
    if (!R.tension) {
        const double c0 = a1 - a2 * R.anpsi, c1 = a2 * (1.0 - R.anpsi), c2 = a2 - a1 * R.anpsi;
        alamb = -(spb[0] * c0 + spb[1] * c1 + spb[2] * c2);
        anpsib += spb[0] * R.alam * a2 + spb[1] * R.alam * a2 + spb[2] * R.alam * a1;
        alamb += depb[0] - R.anpsi * depb[2];
        anpsib += -R.alam * depb[2];
        const double D = a1 - a2 * R.anpsi + a1 * R.anphi * R.anpsi - a2 * R.anphi + 2.0 * sqan * R.hd;
        const double fsb = alamb / D;
        const double Db = -alamb * R.alam / D;
        // fs = sp0 - sp2 anphi + 2 co sqrt(anphi)
        spb[0] += fsb;
        spb[2] += -R.anphi * fsb;
        anphib += fsb * (-R.sp[2] + R.co / sqan);
        cob += fsb * 2.0 * sqan;
        anphib += Db * (a1 * R.anpsi - a2 + R.hd / sqan);
        anpsib += Db * (-a2 + a1 * R.anphi);
        hdb += Db * 2.0 * sqan;
    } else {
        alamb = -(spb[0] * a2 + spb[1] * a2 + spb[2] * a1) + depb[2];
        const double ftb = alamb / a1;  // alam = (sp2 - stc) / a1
        spb[2] += ftb;
        stcb += -ftb;
    }
    // spectral part: A_kk = spb_k, A_kl = B_kl (sq_k - sq_l) / (sp_k - sp_l)
    double A[3][3];
    const double scale = fabs(R.sp[0]) + fabs(R.sp[1]) + fabs(R.sp[2]);
    for (int k = 0; k < 3; k++)
        for (int l = 0; l < 3; l++) {
            if (k == l) {
                A[k][l] = spb[k];
            } else {
                const double ds = R.sp[k] - R.sp[l];
                const double ratio = (fabs(ds) > 1e-13 * scale) ? (R.sq[k] - R.sq[l]) / ds : 1.0;
                A[k][l] = B[k][l] * ratio;
            }
        }
    double S[3][3];
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) {
            double acc = 0.0;
            for (int k = 0; k < 3; k++)
                for (int l = 0; l < 3; l++) acc += R.cn[k][a] * A[k][l] * R.cn[l][b];
            S[a][b] = acc;
        }
    sb_in[0] = S[0][0];
    sb_in[1] = S[1][1];
    sb_in[2] = S[2][2];
    sb_in[3] = S[0][1] + S[1][0];
    sb_in[4] = S[0][2] + S[2][0];
    sb_in[5] = S[1][2] + S[2][1];
}

// ---- the per-tet reverse kernel ------------------------------------------------------------
template <int PLUGIN>
__device__ __forceinline__ void adj_tet_body(const Mesh& m, const Fields& F, const Config& cfg, const AdjState& S,
                                             const AdjBufs& B, int rotate, int first_rev, double dt, int lb) {
    // hooks with a Mohr-Coulomb return map and a plastic strain
    constexpr bool MC = PLUGIN == SNAC_RHEOLOGY_PLASTIC || PLUGIN == SNAC_RHEOLOGY_VISCOPLASTIC;
    TetSlot s = tet_slot(m, lb);
    // corners of step n
    V3 c[4], v[4];
    double T[4];
    long long nid[4];
#pragma unroll
    for (int qn = 0; qn < 4; qn++) {
        if (s.active) {
            nid[qn] = corner_node(m, s.i, s.j, s.k, tet_node_rt(s.t, qn));
            double4 p = S.pos[nid[qn]];
            double4 w = S.vel[nid[qn]];
            c[qn] = {p.x, p.y, p.z};
            T[qn] = p.w;
            v[qn] = {w.x, w.y, w.z};
        } else {
            nid[qn] = 0;
            c[qn] = {qn == 1 ? 1.0 : 0.0, qn == 2 ? 1.0 : 0.0, qn == 3 ? 1.0 : 0.0};
            v[qn] = {0.0, 0.0, 0.0};
            T[qn] = 0.0;
        }
    }
    TetGeom g;
    tet_geometry(c, g);
    // area vectors w_f = n_f A_f (= half the face cross product)
    D3 w[4];
#pragma unroll
    for (int f = 0; f < 4; f++) w[f] = d3(g.n[f].x * g.A[f], g.n[f].y * g.A[f], g.n[f].z * g.A[f]);
    // corner k pairs with face (k+1)%4 in the strain-rate, spin and force sums
    D3 vk[4];
#pragma unroll
    for (int k = 0; k < 4; k++) vk[k] = d3(v[k].x, v[k].y, v[k].z);

    // ---------------- forward recompute --------------------------------------------------
    double s_in[6] = {0, 0, 0, 0, 0, 0};
    if (s.active) {
#pragma unroll
        for (int a = 0; a < 6; a++) s_in[a] = S.stress[s.q * 6 + a];
    }
    double s_pre[6];
#pragma unroll
    for (int a = 0; a < 6; a++) s_pre[a] = s_in[a];
    double s_mid[6];  // stress after each in-place rotation update (for the reverse)
    double r01 = 0, r02 = 0, r12 = 0;
    if (rotate) {
        rotate_stress(v, g, dt, s_pre);
        double r[3];
        spin_rates(v, g, r);  // the same values rotate_stress used
        r01 = r[0];
        r02 = r[1];
        r12 = r[2];
    }
#pragma unroll
    for (int a = 0; a < 6; a++) s_mid[a] = s_pre[a];

    double sr[6];
    tet_strain_rate(v, g, sr);
    double sr_raw[6];
#pragma unroll
    for (int a = 0; a < 6; a++) sr_raw[a] = sr[a];
    const double vsum = grp_sum(g.V, s.base);
    const double VS = 2.0 * (vsum * 0.5);
    const double zVS = recip(VS);
    const double tr1 = dv3(sr[0] + sr[1] + sr[2]);
    const double tr1V = tr1 * g.V;  // the term formed on its own lane, as the forward does
    double P1 = 0.0f;
#pragma unroll
    for (int u = 0; u < NT; u++) P1 += grp(tr1V, s.base, u);
    const double corr1 = -1.0f * tr1 + dvz(P1, VS, zVS);
    sr[0] += corr1;
    sr[1] += corr1;
    sr[2] += corr1;
    double e[6];
#pragma unroll
    for (int a = 0; a < 6; a++) e[a] = sr[a] * dt;

    const int ph = s.active ? phase_of(F, s.e) : 0;
    const DevMaterial& M = F.mats[ph];
    const double cs = (F.coh_scale && s.active) ? F.coh_scale[s.e] : 1.0;
    const double fsc = (F.fric_scale && s.active) ? F.fric_scale[s.e] : 1.0;
    const double vsc = (F.visc_scale && s.active) ? F.visc_scale[s.e] : 1.0;
    double eps_p = (MC && s.active) ? S.eps_p[s.q] : 0.0;
    const double eps_p0 = eps_p;

#if SNAC_ADJ_SMEM_REC
    // the record lives in shared memory (dynamic, one per thread): its ~50
    // doubles then hold no registers between the forward and the reverse
    extern __shared__ __align__(16) unsigned char adj_smem[];
    ConsRec& R = reinterpret_cast<ConsRec*>(adj_smem)[threadIdx.x];
#else
    ConsRec R;
#endif
    double st[6];
#pragma unroll
    for (int a = 0; a < 6; a++) st[a] = s_pre[a];
    R.mx = false;
    if (PLUGIN == SNAC_RHEOLOGY_PLASTIC || PLUGIN == SNAC_RHEOLOGY_ELASTIC) {
        // the elastic trial of the plastic hook and the elastic hook's whole update
        // (the same arithmetic)
        double tr = e[0] + e[1] + e[2];
        st[0] += (2.0f * M.mu) * e[0] + M.lambda * (tr);
        st[1] += (2.0f * M.mu) * e[1] + M.lambda * (tr);
        st[2] += (2.0f * M.mu) * e[2] + M.lambda * (tr);
        st[3] += (2.0f * M.mu) * e[3];
        st[4] += (2.0f * M.mu) * e[4];
        st[5] += (2.0f * M.mu) * e[5];
    } else if (PLUGIN == SNAC_RHEOLOGY_MAXWELL) {
        // maxwell/Constitutive.c:47-184: the trace strain is the volume ratio of the
        // tet (pass n >= 1 rotates: its own volume over the one the previous pass
        // stored; pass 0 reads both as the state holds them), the second invariant
        // includes the shear strains, and only phase 0 takes the update
        R.mx = (ph == 0);
        R.trs = st[0] + st[1] + st[2];
        R.vcur = rotate ? g.V : (s.active ? S.vol[s.q * 2 + 0] : 1.0);
        R.vold = s.active ? S.vol[s.q * 2 + (rotate ? 0 : 1)] : 1.0;
        R.tre = dv(R.vcur, R.vold) - 1.0f;
        const double tn3 = dv3(R.tre), ts3 = dv3(R.trs);
        for (int a = 0; a < 3; a++) R.d[a] = e[a] - tn3;
        for (int a = 0; a < 3; a++) R.sd[a] = st[a] - ts3;
        R.Q = R.d[1] * R.d[2] + R.d[2] * R.d[0] + R.d[0] * R.d[1] - e[3] * e[3] - e[4] * e[4] - e[5] * e[5];
        double J = sqrt(fabs(R.Q)) / dt;
        R.J_from_sqrt = !(J == 0.0f);
        if (J == 0.0f) J = M.refsrate;
        R.J = J;
        double avgTemp = 0.0;
        for (int qn = 0; qn < 4; qn++) avgTemp += 0.25 * T[qn];
        const double eta = arrhenius_viscosity(M, M.refvisc, J, avgTemp);
        R.eta_free = (eta > M.vis_min && eta < M.vis_max);
        R.eta = eta;
        R.eta_base = 0.0;
        R.tmp = dv(M.mu, 2.0f * (eta)) * dt;
        R.vic1 = 1.0f - R.tmp;
        R.vic2 = dv(1.0f, 1.0f + R.tmp);
        if (R.mx) {
            const double bulkm = M.lambda + dv3(2.0f * M.mu);
            double stressd[3] = {R.sd[0], R.sd[1], R.sd[2]};
            maxwell_update(st, e, stressd, R.d, ts3, R.tre, M.mu, eta, dt, bulkm);
        }
    } else {
        const double bulkm = M.lambda + dv3(2.0f * M.mu);
        R.trs = st[0] + st[1] + st[2];
        R.tre = e[0] + e[1] + e[2];
        for (int a = 0; a < 3; a++) R.d[a] = e[a] - dv3(R.tre);
        for (int a = 0; a < 3; a++) R.sd[a] = st[a] - dv3(R.trs);
        R.Q = R.d[1] * R.d[2] + R.d[2] * R.d[0] + R.d[0] * R.d[1];
        double J = sqrt(fabs(R.Q)) / dt;
        R.J_from_sqrt = !(J == 0.0f);
        if (J == 0.0f) J = M.refsrate;
        R.J = J;
        double avgTemp = 0.0;
        for (int qn = 0; qn < 4; qn++) avgTemp += 0.25 * T[qn];
        const double refvisc = M.refvisc * vsc;
        // unclipped viscosity without the element's scale: d eta / d scale
        R.eta_base = arrhenius_base(M, M.refvisc, J, avgTemp);
        double eta = arrhenius_viscosity(M, refvisc, J, avgTemp);
        R.eta_free = (eta > M.vis_min && eta < M.vis_max);
        R.eta = eta;
        R.tmp = dv(M.mu, 2.0f * (eta)) * dt;
        R.vic1 = 1.0f - R.tmp;
        R.vic2 = dv(1.0f, 1.0f + R.tmp);
        double stressd[3] = {R.sd[0], R.sd[1], R.sd[2]};
        maxwell_update(st, e, stressd, R.d, dv3(R.trs), R.tre, M.mu, eta, dt, bulkm);
    }
    const double a1 = M.lambda + 2.0f * M.mu;
    const double a2 = M.lambda;
    R.yield = false;
    R.tension = false;
    R.alam = 0.0;
    R.inc = 0.0;
    R.co = R.hd = R.fa = R.da = R.fa_b = R.co_b = R.tgf_b = R.tgc_b = R.tgd = 0.0;
    R.sphi = R.spsi = R.anphi = R.anpsi = R.stc = 0.0;
    R.dpl = 1.0;
    R.clamped = false;
    R.stc_from_co = false;
    if (MC) {
        // softening lookup: this tet's own segment (plastic: first match, clamp past the end;
        // visco-plastic: last match)
        bool matched = false;
        for (int i = 0; i < M.nsegments; i++) {
            const double pl1 = M.plstrain[i];
            const double pl2 = M.plstrain[i + 1];
            if (eps_p >= pl1 && eps_p <= pl2) {
                const double dpl = pl2 - pl1;
                R.dpl = dpl;
                double tg[3] = {M.fric[i + 1] - M.fric[i], M.coh[i + 1] - M.coh[i], M.dil[i + 1] - M.dil[i]};
                dvz_n(tg, dpl, M.zpl[i]);
                R.tgf_b = tg[0];
                R.tgc_b = tg[1];
                R.tgd = tg[2];
                R.fa_b = M.fric[i] + R.tgf_b * (eps_p - pl1);
                R.co_b = M.coh[i] + R.tgc_b * (eps_p - pl1);
                R.da = M.dil[i] + R.tgd * (eps_p - pl1);
                matched = true;
                R.clamped = false;
                if (PLUGIN == SNAC_RHEOLOGY_PLASTIC) break;
            } else if (PLUGIN == SNAC_RHEOLOGY_PLASTIC && i == M.nsegments - 1 && eps_p > pl2) {
                R.fa_b = M.fric[M.nsegments];
                R.co_b = M.coh[M.nsegments];
                R.da = M.dil[M.nsegments];
                R.tgf_b = R.tgc_b = R.tgd = 0.0;
                matched = true;
                R.clamped = true;
                break;
            }
        }
        if (s.active && !matched) report(F.sc, SNAC_GPU_ENOTSUP, s.e);  // the carried-over lookup is not differentiated
        // values as the forward forms them (scales applied to the table entries)
        {
            // recompute exactly as the forward does, for identical branch decisions
            double fa = 0.0, co = 0.0, hd = 0.0;
            for (int i = 0; i < M.nsegments; i++) {
                const double pl1 = M.plstrain[i];
                const double pl2 = M.plstrain[i + 1];
                double f0 = F.fric_scale ? M.fric[i] * fsc : M.fric[i];
                double f1 = F.fric_scale ? M.fric[i + 1] * fsc : M.fric[i + 1];
                double c0 = F.coh_scale ? M.coh[i] * cs : M.coh[i];
                double c1 = F.coh_scale ? M.coh[i + 1] * cs : M.coh[i + 1];
                if (eps_p >= pl1 && eps_p <= pl2) {
                    double tg[2] = {f1 - f0, c1 - c0};
                    dvz_n(tg, pl2 - pl1, M.zpl[i]);
                    const double tgf = tg[0], tgc = tg[1];
                    fa = f0 + tgf * (eps_p - pl1);
                    co = c0 + tgc * (eps_p - pl1);
                    hd = tgc;
                    if (PLUGIN == SNAC_RHEOLOGY_PLASTIC) break;
                } else if (PLUGIN == SNAC_RHEOLOGY_PLASTIC && i == M.nsegments - 1 && eps_p > pl2) {
                    fa = F.fric_scale ? M.fric[M.nsegments] * fsc : M.fric[M.nsegments];
                    co = F.coh_scale ? M.coh[M.nsegments] * cs : M.coh[M.nsegments];
                    hd = 0.0;
                    break;
                }
            }
            R.fa = fa;
            R.co = co;
            R.hd = hd;
        }
        const bool phi_ok = (PLUGIN == SNAC_RHEOLOGY_PLASTIC) ? (R.fa >= 0.0f) : (R.fa > 0.0f);
        if (s.active && !phi_ok) report(F.sc, SNAC_GPU_ENOTSUP, s.e);
        R.stc = M.ten_off;
        R.stc_from_co = false;
        // constant-angle values as the forward takes them (host-evaluated, same bits)
        const bool fconst = M.fric_const && R.fa == M.fric0;
        if (R.fa > 0.0) {
            double tmp = fconst ? dvz(R.co, M.tan_fric0, M.ztan_fric0) : dv(R.co, tan_fric(M, R.fa));
            if (tmp < R.stc) {
                R.stc = tmp;
                R.stc_from_co = true;
            }
        }
        R.sphi = sin_fric(M, R.fa);
        R.spsi = sin_dil(M, R.da);
        R.anphi = fconst ? M.anphi0 : dv(1.0f + R.sphi, 1.0f - R.sphi);
        R.anpsi = (M.dil_const && R.da == M.dil0) ? M.anpsi0 : dv(1.0f + R.spsi, 1.0f - R.spsi);
        double st_trial[6];
#pragma unroll
        for (int a = 0; a < 6; a++) st_trial[a] = st[a];
        if (!surely_elastic(st, R.co, R.anphi, fconst ? M.sq_anphi0 : sqrt(R.anphi), R.stc)) {
            principal_stresses(st, R.sp, R.cn);
            double sp[3] = {R.sp[0], R.sp[1], R.sp[2]};
            double fs = sp[0] - sp[2] * R.anphi + 2 * R.co * sqrt(R.anphi);
            double ft = sp[2] - R.stc;
            double aP = sqrt(1.0f + R.anphi * R.anphi) + R.anphi;
            double sP = R.stc * R.anphi - 2 * R.co * sqrt(R.anphi);
            double hh = sp[2] - R.stc + aP * (sp[0] - sP);
            R.tension = !(hh < 0.0f);
            const double ep_before = eps_p;
            R.yield = mc_return_map(sp, R.cn, st, eps_p, R.co, R.hd, R.anphi, R.anpsi, R.stc, a1, a2) != 0;
            (void)fs;
            (void)ft;
            if (R.yield) {
                R.alam = R.tension ? dv(ft, a1)
                                   : dv(fs, a1 - a2 * R.anpsi + a1 * R.anphi * R.anpsi - a2 * R.anphi +
                                                2.0 * sqrt(R.anphi) * R.hd);
                R.inc = eps_p - ep_before;
                for (int k = 0; k < 3; k++) R.sq[k] = sp[k];
            }
        }
    }
    // stress averaging over the hex
    const double trS = dv3(st[0] + st[1] + st[2]);
    const double trSV = trS * g.V;
    double P2 = 0.0f;
#pragma unroll
    for (int u = 0; u < NT; u++) P2 += grp(trSV, s.base, u);
    const double corr2 = -1.0f * trS + dvz(P2, VS, zVS);
    double sa[6];
#pragma unroll
    for (int a = 0; a < 6; a++) sa[a] = st[a];
    sa[0] += corr2;
    sa[1] += corr2;
    sa[2] += corr2;

    // ---------------- reverse ----------------------------------------------------------------
    // The reverse sweep needs no reference rounding: divisions by constants and
    // by the tet volume are multiplications by reciprocals.
    constexpr double K16 = 1.0 / 6.0, K13 = 1.0 / 3.0;
    const double iVS = zVS, i9V = (1.0 / 9.0) * g.zV, i3V = K13 * g.zV, i6V = K16 * g.zV;
    D3 wb[4] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    D3 vb[4] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    double Vb = 0.0;
    double sab[6] = {0, 0, 0, 0, 0, 0};
    if (s.active && !first_rev) {
#pragma unroll
        for (int a = 0; a < 6; a++) sab[a] = B.sbar[s.q * 6 + a];
    }
    // Force: node k takes sigma . w_{(k+1)%4} / 6, -g rho V / 8 in y, and the inertial mass
    // of face (k+1)%4 (constant dt: (lambda + 2 mu) max_d w_d^2 / (9 V) dt^2)
    const double rho = M.density;
    const double alpha1 = (M.lambda + 2.0f * M.mu);
    if (s.active) {
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int f = (k + 1) & 3;
            const double4 fb = B.fbar[nid[k]];
            const D3& wf = w[f];
            sab[0] += fb.x * wf.x * K16;
            sab[1] += fb.y * wf.y * K16;
            sab[2] += fb.z * wf.z * K16;
            sab[3] += (fb.x * wf.y + fb.y * wf.x) * K16;
            sab[4] += (fb.x * wf.z + fb.z * wf.x) * K16;
            sab[5] += (fb.y * wf.z + fb.z * wf.y) * K16;
            wb[f].x += (sa[0] * fb.x + sa[3] * fb.y + sa[4] * fb.z) * K16;
            wb[f].y += (sa[3] * fb.x + sa[1] * fb.y + sa[5] * fb.z) * K16;
            wb[f].z += (sa[4] * fb.x + sa[5] * fb.y + sa[2] * fb.z) * K16;
            Vb += -cfg.gravity * rho / 8.0 * fb.y;
            // inertial mass of face f
            int dstar = 0;
            double best = wf.x * wf.x;
            if (wf.y * wf.y > best) {
                best = wf.y * wf.y;
                dstar = 1;
            }
            if (wf.z * wf.z > best) {
                best = wf.z * wf.z;
                dstar = 2;
            }
            const double mf = alpha1 * best * i9V * (dt * dt);
            addc(wb[f], dstar, fb.w * alpha1 * 2.0 * cmp(wf, dstar) * i9V * (dt * dt));
            Vb += -fb.w * mf * g.zV;
        }
    }
    // trace averaging: sa_dd = st_dd - trS + P2 / VS
    double stb[6];
#pragma unroll
    for (int a = 0; a < 6; a++) stb[a] = sab[a];
    const double c2b = sab[0] + sab[1] + sab[2];
    const double P2b_own = c2b * iVS;  // summed over the hex below
    const double P2b = grp_sum(s.active ? P2b_own : 0.0, s.base);
    double VSb = -(P2 * (iVS * iVS)) * grp_sum(s.active ? c2b : 0.0, s.base);
    double trSb = -c2b + P2b * g.V;
    Vb += P2b * trS;
    stb[0] += trSb * K13;
    stb[1] += trSb * K13;
    stb[2] += trSb * K13;

    // constitutive reverse: MC return map
    double epb = (s.active && !first_rev) ? B.epbar[s.q] : 0.0;  // adjoint of eps_p^{n+1}
    double cob = 0.0, hdb = 0.0, anphib = 0.0, anpsib = 0.0, stcb = 0.0;
    double trialb[6];
    if (R.yield) {
        mc_reverse(R, stb, epb, a1, a2, trialb, cob, hdb, anphib, anpsib, stcb);
    } else {
#pragma unroll
        for (int a = 0; a < 6; a++) trialb[a] = stb[a];
    }
    // softening chain: anphi(sphi(fa)), anpsi(spsi(da)), stc(co, fa)
    const double deg = degrad();
    double fab = 0.0, dab = 0.0;
    if (MC) {
        const double dan = 2.0 / ((1.0 - R.sphi) * (1.0 - R.sphi));
        fab += anphib * dan * cos(R.fa * deg) * deg;
        const double dap = 2.0 / ((1.0 - R.spsi) * (1.0 - R.spsi));
        dab += anpsib * dap * cos(R.da * deg) * deg;
        if (R.stc_from_co) {
            const double tn = tan(R.fa * deg);
            const double cs2 = cos(R.fa * deg);
            cob += stcb / tn;
            fab += stcb * (-R.co / (tn * tn)) * (deg / (cs2 * cs2));
        }
    }
    // co = cs * co_b(eps_p), hd = cs * tgc_b, fa = fsc * fa_b(eps_p), da(eps_p)
    double csb = cob * R.co_b + hdb * R.tgc_b;
    double fscb = fab * R.fa_b;
    epb += cob * cs * R.tgc_b + fab * fsc * R.tgf_b + dab * R.tgd;
    double vscb = 0.0;

    // elastic trial (plastic), elastic update, or Maxwell step (Maxwell, visco-plastic)
    double sprb[6], eb[6];
    double Vcb = 0.0, Vob = 0.0;  // Maxwell: adjoints of the current and the old tet volume
    if (PLUGIN == SNAC_RHEOLOGY_PLASTIC || PLUGIN == SNAC_RHEOLOGY_ELASTIC) {
#pragma unroll
        for (int a = 0; a < 6; a++) sprb[a] = trialb[a];
        const double lsum = trialb[0] + trialb[1] + trialb[2];
        for (int a = 0; a < 3; a++) eb[a] = 2.0 * M.mu * trialb[a] + M.lambda * lsum;
        for (int a = 3; a < 6; a++) eb[a] = 2.0 * M.mu * trialb[a];
    } else if (PLUGIN == SNAC_RHEOLOGY_MAXWELL) {
        if (!R.mx) {
#pragma unroll
            for (int a = 0; a < 6; a++) {
                sprb[a] = trialb[a];
                eb[a] = 0.0;
            }
        } else {
            const double bulkm = M.lambda + 2.0 * M.mu * K13;
            const double mu = M.mu;
            double sdb[3], db[3] = {0, 0, 0};
            double vic1b = 0.0, vic2b = 0.0;
            const double osum = trialb[0] + trialb[1] + trialb[2];
            double trsb = osum * K13, treb = bulkm * osum;
            for (int a = 0; a < 3; a++) {
                const double sdo = trialb[a];
                sdb[a] = sdo * R.vic1 * R.vic2;
                db[a] += sdo * 2.0 * mu * R.vic2;
                vic1b += sdo * R.sd[a] * R.vic2;
                vic2b += sdo * (R.sd[a] * R.vic1 + 2.0 * mu * R.d[a]);
            }
            for (int a = 3; a < 6; a++) {
                sprb[a] = trialb[a] * R.vic1 * R.vic2;
                eb[a] = trialb[a] * 2.0 * mu * R.vic2;
                vic1b += trialb[a] * s_pre[a] * R.vic2;
                vic2b += trialb[a] * (s_pre[a] * R.vic1 + 2.0 * mu * e[a]);
            }
            const double tmpb = -vic1b - vic2b * R.vic2 * R.vic2;
            const double etab = -tmpb * R.tmp / R.eta;
            if (R.eta_free && R.J_from_sqrt) {
                const double p = 1.0 / M.srexponent - 1.0;
                const double Jb = etab * R.eta * p / R.J;
                const double Qb = Jb * sgnd(R.Q) / (2.0 * sqrt(fabs(R.Q)) * dt);
                db[0] += Qb * (R.d[2] + R.d[1]);
                db[1] += Qb * (R.d[2] + R.d[0]);
                db[2] += Qb * (R.d[1] + R.d[0]);
                for (int a = 3; a < 6; a++) eb[a] += Qb * (-2.0 * e[a]);
            }
            for (int a = 0; a < 3; a++) {
                eb[a] = db[a];
                treb -= db[a] * K13;
                sprb[a] = sdb[a];
                trsb -= sdb[a] * K13;
            }
            for (int a = 0; a < 3; a++) sprb[a] += trsb;
            // tre = vcur / vold - 1
            Vcb = treb / R.vold;
            Vob = -treb * R.vcur / (R.vold * R.vold);
        }
    } else {
        const double bulkm = M.lambda + 2.0 * M.mu * K13;
        const double mu = M.mu;
        double sdb[3], db[3] = {0, 0, 0};
        double vic1b = 0.0, vic2b = 0.0;
        const double VSb2 = trialb[0] + trialb[1] + trialb[2];
        double trsb = VSb2 * K13, treb = bulkm * VSb2;
        for (int a = 0; a < 3; a++) {
            const double sdo = trialb[a];
            sdb[a] = sdo * R.vic1 * R.vic2;
            db[a] += sdo * 2.0 * mu * R.vic2;
            vic1b += sdo * R.sd[a] * R.vic2;
            vic2b += sdo * (R.sd[a] * R.vic1 + 2.0 * mu * R.d[a]);
        }
        for (int a = 3; a < 6; a++) {
            sprb[a] = trialb[a] * R.vic1 * R.vic2;
            eb[a] = trialb[a] * 2.0 * mu * R.vic2;
            vic1b += trialb[a] * s_pre[a] * R.vic2;
            vic2b += trialb[a] * (s_pre[a] * R.vic1 + 2.0 * mu * e[a]);
        }
        const double tmpb = -vic1b - vic2b * R.vic2 * R.vic2;
        const double etab = -tmpb * R.tmp / R.eta;
        if (R.eta_free) {
            vscb += etab * R.eta_base;
            if (R.J_from_sqrt) {
                const double p = 1.0 / M.srexponent - 1.0;
                const double Jb = etab * R.eta * p / R.J;
                const double Qb = Jb * sgnd(R.Q) / (2.0 * sqrt(fabs(R.Q)) * dt);
                db[0] += Qb * (R.d[2] + R.d[1]);
                db[1] += Qb * (R.d[2] + R.d[0]);
                db[2] += Qb * (R.d[1] + R.d[0]);
            }
        }
        for (int a = 0; a < 3; a++) {
            eb[a] = db[a];
            treb -= db[a] * K13;
            sprb[a] = sdb[a];
            trsb -= sdb[a] * K13;
        }
        for (int a = 0; a < 3; a++) {
            sprb[a] += trsb;
            eb[a] += treb;
        }
    }
    // strain rate: e = sr dt, sr_dd = sr_raw_dd + corr1
    double srb[6];
#pragma unroll
    for (int a = 0; a < 6; a++) srb[a] = eb[a] * dt;
    const double c1b = srb[0] + srb[1] + srb[2];
    const double P1b = grp_sum(s.active ? c1b * iVS : 0.0, s.base);
    VSb += -(P1 * (iVS * iVS)) * grp_sum(s.active ? c1b : 0.0, s.base);
    const double tr1b = -c1b + P1b * g.V;
    Vb += P1b * tr1;
    srb[0] += tr1b * K13;
    srb[1] += tr1b * K13;
    srb[2] += tr1b * K13;
    // raw strain rate: sr_d = -S_dd / (3V), sr_ab = -(S_ab + S_ba) / (6V), S_ab = sum_k v_k,a w_k,b
    {
        double Sb[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        for (int d = 0; d < 3; d++) Sb[d][d] = -srb[d] * i3V;
        Sb[0][1] = Sb[1][0] = -srb[3] * i6V;
        Sb[0][2] = Sb[2][0] = -srb[4] * i6V;
        Sb[1][2] = Sb[2][1] = -srb[5] * i6V;
        for (int a = 0; a < 6; a++) Vb += srb[a] * (-sr_raw[a] * g.zV);
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const D3& wk = w[(k + 1) & 3];
            for (int a = 0; a < 3; a++)
                for (int b = 0; b < 3; b++) {
                    addc(vb[k], a, Sb[a][b] * cmp(wk, b));
                    addc(wb[(k + 1) & 3], b, Sb[a][b] * cmp(vk[k], a));
                }
        }
    }
    // rotation of step n-1: s_pre = Rot(s_in, r, dt), in place, in the forward's order
    double sinb[6];
#pragma unroll
    for (int a = 0; a < 6; a++) sinb[a] = sprb[a];
    if (rotate) {
        // values each statement read: statement i reads the already-updated entries < i
        const double* si = s_in;
        const double* sf = s_mid;
        double r01b = 0, r02b = 0, r12b = 0;
        double* b = sinb;
        // 6: s5 += dt r12 (s2 - s1) + dt (-r01 s4 - r02 s3)
        b[2] += b[5] * dt * r12;
        b[1] -= b[5] * dt * r12;
        b[4] += -b[5] * dt * r01;
        b[3] += -b[5] * dt * r02;
        r12b += b[5] * dt * (sf[2] - sf[1]);
        r01b += -b[5] * dt * sf[4];
        r02b += -b[5] * dt * sf[3];
        // 5: s4 += dt r02 (s2 - s0) + dt (r01 s5 - r12 s3)
        b[2] += b[4] * dt * r02;
        b[0] -= b[4] * dt * r02;
        b[5] += b[4] * dt * r01;
        b[3] -= b[4] * dt * r12;
        r02b += b[4] * dt * (sf[2] - sf[0]);
        r01b += b[4] * dt * si[5];
        r12b += -b[4] * dt * sf[3];
        // 4: s3 += dt r01 (s1 - s0) + dt (r02 s5 + r12 s4)
        b[1] += b[3] * dt * r01;
        b[0] -= b[3] * dt * r01;
        b[5] += b[3] * dt * r02;
        b[4] += b[3] * dt * r12;
        r01b += b[3] * dt * (sf[1] - sf[0]);
        r02b += b[3] * dt * si[5];
        r12b += b[3] * dt * si[4];
        // 3: s2 += 2 dt (-r02 s4 - r12 s5)
        b[4] += -2.0 * dt * r02 * b[2];
        b[5] += -2.0 * dt * r12 * b[2];
        r02b += -2.0 * dt * si[4] * b[2];
        r12b += -2.0 * dt * si[5] * b[2];
        // 2: s1 += 2 dt (-r01 s3 + r12 s5)
        b[3] += -2.0 * dt * r01 * b[1];
        b[5] += 2.0 * dt * r12 * b[1];
        r01b += -2.0 * dt * si[3] * b[1];
        r12b += 2.0 * dt * si[5] * b[1];
        // 1: s0 += 2 dt (r01 s3 + r02 s4)
        b[3] += 2.0 * dt * r01 * b[0];
        b[4] += 2.0 * dt * r02 * b[0];
        r01b += 2.0 * dt * si[3] * b[0];
        r02b += 2.0 * dt * si[4] * b[0];
        // r_ab = -SP_ab / (6 V), SP_ab = sum_k (v_k,a w_k,b - v_k,b w_k,a)
        const double rr[3] = {r01, r02, r12};
        const double rb[3] = {r01b, r02b, r12b};
        const int pa[3] = {0, 0, 1}, pb[3] = {1, 2, 2};
        for (int r = 0; r < 3; r++) {
            const double SPb = -rb[r] * i6V;
            Vb += rb[r] * (-rr[r] * g.zV);
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const D3& wk = w[(k + 1) & 3];
                addc(vb[k], pa[r], SPb * cmp(wk, pb[r]));
                addc(vb[k], pb[r], -SPb * cmp(wk, pa[r]));
                addc(wb[(k + 1) & 3], pb[r], SPb * cmp(vk[k], pa[r]));
                addc(wb[(k + 1) & 3], pa[r], -SPb * cmp(vk[k], pb[r]));
            }
        }
    }
    // VS = sum over the hex of V; VSb already holds the hex total (both terms
    // were summed over the hex), so every tet's V receives it once
    Vb += VSb;
    if (PLUGIN == SNAC_RHEOLOGY_MAXWELL && rotate) {
        // a rotating pass stores its own volume, which the next pass reads as the old one
        if (s.active && !first_rev) Vb += B.vobar[s.q];
        Vb += Vcb;
    }

    // geometry: V = |det(c1-c0, c2-c0, c3-c0)| / 6, w_f = ((c_f1 - c_f0) x (c_f2 - c_f0)) / 2
    D3 cb[4] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    D3 C[4];
#pragma unroll
    for (int k = 0; k < 4; k++) C[k] = d3(c[k].x, c[k].y, c[k].z);
    {
        const D3 x2 = C[1] - C[0], x3 = C[2] - C[0], x4 = C[3] - C[0];
        const double det = dot(x4, cross(x2, x3));
        const double detb = Vb * sgnd(det) * K16;
        const D3 g2 = detb * cross(x3, x4), g3 = detb * cross(x4, x2), g4 = detb * cross(x2, x3);
        cb[1] = cb[1] + g2;
        cb[2] = cb[2] + g3;
        cb[3] = cb[3] + g4;
        cb[0] = cb[0] - (g2 + g3 + g4);
    }
#pragma unroll
    for (int f = 0; f < 4; f++) {
        const int f0 = face_node(f, 0), f1 = face_node(f, 1), f2 = face_node(f, 2);
        const D3 u = C[f1] - C[f0], vv = C[f2] - C[f0];
        const D3 Pb = 0.5 * wb[f];
        const D3 ub = cross(vv, Pb), vvb = cross(Pb, u);
        cb[f1] = cb[f1] + ub;
        cb[f2] = cb[f2] + vvb;
        cb[f0] = cb[f0] - (ub + vvb);
    }

    if (s.active) {
        // tet-major rows, as the forward's force terms: the node gather reads
        // one row at consecutive hexes
        const long long R = m.ner;
        double* o = B.cbuf + (long long)(s.t * 24) * R + s.e;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            o[(k * 6 + 0) * R] = cb[k].x;
            o[(k * 6 + 1) * R] = cb[k].y;
            o[(k * 6 + 2) * R] = cb[k].z;
            o[(k * 6 + 3) * R] = vb[k].x;
            o[(k * 6 + 4) * R] = vb[k].y;
            o[(k * 6 + 5) * R] = vb[k].z;
        }
        // pass 0 leaves the adjoint of the stress the state held
#pragma unroll
        for (int a = 0; a < 6; a++) B.sbar[s.q * 6 + a] = sinb[a];
        if (PLUGIN == SNAC_RHEOLOGY_MAXWELL) B.vobar[s.q] = rotate ? Vob : 0.0;
        B.epbar[s.q] = epb;
        B.pbar[s.q * 3 + 0] += csb;
        B.pbar[s.q * 3 + 1] += fscb;
        B.pbar[s.q * 3 + 2] += vscb;
    }
    (void)eps_p0;
}

#ifndef SNAC_ADJ_MINB
#define SNAC_ADJ_MINB 1  // resident blocks per SM asked of k_adj_tet
#endif
template <int PLUGIN>
__global__ void __launch_bounds__(ELEM_WARPS * 32, SNAC_ADJ_MINB) k_adj_tet(Mesh m, Fields F, Config cfg, AdjState S, AdjBufs B,
                                                             int rotate, int first_rev, double dt) {
    adj_tet_body<PLUGIN>(m, F, cfg, S, B, rotate, first_rev, dt, blockIdx.x);
}

// Node adjoints: gather the corner adjoints of tet pass n (fixed order), then
// the reverse of the node update of step n-1:
//   x^n = x^{n-1} + dt v^n,  v^n_c = v^{n-1}_c + dt F_d,c / m  (free components)
//   F_d = F (1 - demf sgn(v^{n-1}) sgn(F))
// cur = S^n (its force holds F_d and m of step n-1), prev = S^{n-1} (velocities).
__global__ void __launch_bounds__(128) k_adj_nodes(Mesh m, Fields F, AdjState cur, AdjState prev, AdjBufs B,
                                                   int gather, int update, double dt, double demf) {
    long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= m.nn) return;
    double4 xb = B.xbar[n], vb = B.vbar[n];
    if (gather) {
        int i, j, k;
        split3(n, m.nnx, m.nny, i, j, k);
        for (int ne = 0; ne < 8; ne++) {
            int ei = i - 1 + (ne & 1), ej = j - 1 + ((ne >> 1) & 1), ek = k - 1 + ((ne >> 2) & 1);
            if (ei < 0 || ej < 0 || ek < 0 || ei >= m.nx || ej >= m.ny || ek >= m.nz) continue;
            long long e = (long long)ei + (long long)ej * m.nx + (long long)ek * m.nx * m.ny;
            for (int idx = 0; idx < 5; idx++) {
                const int t = node_tet(ne, idx);
                const int qn = (node_face(ne, idx) + 3) & 3;  // face f is opposite local node (f+3)%4
                const long long R = m.ner;
                const double* o = B.cbuf + (long long)(t * 24 + qn * 6) * R + e;
                xb.x += o[0];
                xb.y += o[R];
                xb.z += o[2 * R];
                vb.x += o[3 * R];
                vb.y += o[4 * R];
                vb.z += o[5 * R];
            }
        }
    }
    if (update) {
        vb.x += dt * xb.x;
        vb.y += dt * xb.y;
        vb.z += dt * xb.z;
        const double4 fd = cur.force[n];
        const double4 vp = prev.vel[n];
        const uchar4 bc = F.bc[n];
        const double mass = fd.w;
        double fb[3], mb = 0.0;
        const double vbc[3] = {vb.x, vb.y, vb.z};
        const double fdc[3] = {fd.x, fd.y, fd.z};
        const double vpc[3] = {vp.x, vp.y, vp.z};
        const bool fixed[3] = {bc.x != 255, bc.y != 255, bc.z != 255};
        double vout[3];
        const double im = 1.0 / mass;
        for (int c = 0; c < 3; c++) {
            if (fixed[c]) {
                fb[c] = 0.0;
                vout[c] = 0.0;
            } else {
                const double fdb = vbc[c] * dt * im;
                mb += -vbc[c] * dt * fdc[c] * (im * im);
                fb[c] = fdb * (1.0 - demf * sgnd(vpc[c]) * sgnd(fdc[c]));
                vout[c] = vbc[c];
            }
        }
        B.fbar[n] = make_double4(fb[0], fb[1], fb[2], mb);
        vb = make_double4(vout[0], vout[1], vout[2], 0.0);
    }
    B.xbar[n] = xb;
    B.vbar[n] = vb;
}

// loss on the top surface (j = nny - 1): per node w_v (v_y - tv)^2 + w_h (y - ty)^2,
// its gradient seeds the adjoints; every other node's adjoint starts at zero
__global__ void k_adj_loss(Mesh m, const double4* pos, const double4* vel, const double* tv, const double* ty,
                           double wv, double wh, double* terms, AdjBufs B) {
    long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= m.nn) return;
    int i, j, k;
    split3(n, m.nnx, m.nny, i, j, k);
    double4 xb = make_double4(0, 0, 0, 0), vb = make_double4(0, 0, 0, 0);
    if (j == m.nny - 1) {
        long long t = (long long)i + (long long)k * m.nnx;
        const double dv_ = vel[n].y - tv[t], dy = pos[n].y - ty[t];
        terms[t] = wv * dv_ * dv_ + wh * dy * dy;
        vb.y = 2.0 * wv * dv_;
        xb.y = 2.0 * wh * dy;
    }
    B.xbar[n] = xb;
    B.vbar[n] = vb;
    B.fbar[n] = make_double4(0, 0, 0, 0);
}

// up to 6 array copies in one launch (checkpoint save / restore), 64-bit words
struct CopyJob {
    unsigned long long* dst[7];
    const unsigned long long* src[7];
    long long n[7];
    int count;
};
__global__ void __launch_bounds__(256) k_copy_many(CopyJob J) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (int a = 0; a < J.count; a++) {
        unsigned long long* d = J.dst[a];
        const unsigned long long* s = J.src[a];
        for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < J.n[a]; i += stride) d[i] = s[i];
    }
}

// per-element gradients: sum of the element's 10 tets in tet order
__global__ void k_adj_reduce(long long ne, const double* pbar, double* gc, double* gf, double* gv) {
    long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ne) return;
    double a = 0, b = 0, c = 0;
    for (int t = 0; t < NT; t++) {
        a += pbar[(e * NT + t) * 3 + 0];
        b += pbar[(e * NT + t) * 3 + 1];
        c += pbar[(e * NT + t) * 3 + 2];
    }
    gc[e] = a;
    gf[e] = b;
    gv[e] = c;
}

}  // namespace snac
