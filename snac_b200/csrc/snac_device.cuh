// snac_device.cuh — device-side building blocks of the SNAC step for sm_100a.
//
// Everything here is FP64.  The translation unit that includes this file is
// compiled with -fmad=false, so every expression below rounds exactly like
// the reference's x86-64 build (no FMA contraction, IEEE division and square
// root); the expressions keep the reference's evaluation order, and each
// function cites the reference lines it computes.  Paths are relative to the
// SNAC source tree.
#pragma once

#include <cstdint>
#include <cstring>
#include <cmath>

#include "snac_gpu.h"

namespace snac {

constexpr int NT = 10;        // Tetrahedra_Count
// Kernel instances of the visco-plastic hook for models with a
// Drucker-Prager phase (the extra state and branch stay out of the
// Mohr-Coulomb instances' registers).
constexpr int SNAC_VP_DP = SNAC_RHEOLOGY_VISCOPLASTIC | 0x100;
__host__ __device__ constexpr bool is_vp(int plugin) { return (plugin & SNAC_RHEOLOGY_VISCOPLASTIC) != 0; }
constexpr int MAX_PHASES = SNAC_MAX_PHASES;

// TetrahedraTables.c:42-84 (tets 0-4 are the first five-tet set, 5-9 the second).
// Face f of a tet is the triangle opposite its local node (3,0,1,2)[f].
// The tables are compile-time functions: inside unrolled loops every index
// folds to a constant and the corner coordinates stay in registers.
__host__ __device__ constexpr int tet_node(int t, int q) {
    constexpr int tab[NT][4] = {{7, 2, 3, 0}, {0, 5, 4, 7}, {2, 5, 1, 0}, {5, 2, 6, 7}, {2, 5, 0, 7},
                                {3, 4, 7, 6}, {4, 3, 0, 1}, {6, 1, 2, 3}, {1, 6, 5, 4}, {1, 3, 6, 4}};
    return tab[t][q];
}
__host__ __device__ constexpr int face_node(int f, int k) {
    constexpr int tab[4][3] = {{0, 1, 2}, {1, 3, 2}, {0, 2, 3}, {3, 1, 0}};
    return tab[f][k];
}
__host__ __device__ constexpr int node_tet(int ne, int i) {
    constexpr int tab[8][5] = {{3, 5, 7, 8, 9}, {0, 1, 3, 4, 5}, {1, 2, 3, 4, 8}, {1, 5, 6, 8, 9},
                               {0, 2, 3, 4, 7}, {0, 5, 6, 7, 9}, {2, 6, 7, 8, 9}, {0, 1, 2, 4, 6}};
    return tab[ne][i];
}
__host__ __device__ constexpr int node_face(int ne, int i) {
    constexpr int tab[8][5] = {{3, 0, 1, 2, 3}, {1, 0, 0, 0, 3}, {2, 2, 1, 2, 3}, {3, 2, 1, 0, 0},
                               {2, 1, 2, 1, 3}, {3, 1, 2, 0, 2}, {3, 0, 2, 1, 1}, {0, 1, 0, 3, 3}};
    return tab[ne][i];
}
// element-local corner -> (di,dj,dk), HexaEL.c:456-471: corners 1,2,5,6 have di=1 ...
__host__ __device__ constexpr int corner_di(int c) { return (c == 1 || c == 2 || c == 5 || c == 6) ? 1 : 0; }
__host__ __device__ constexpr int corner_dj(int c) { return (c == 2 || c == 3 || c == 6 || c == 7) ? 1 : 0; }
__host__ __device__ constexpr int corner_dk(int c) { return c >= 4 ? 1 : 0; }

// tet_node for a per-lane (run-time) tet index, from two packed 64-bit words
// (3 bits per corner): no constant-memory lookups that would serialise.
__host__ __device__ constexpr unsigned long long pack_tets(int t0) {
    unsigned long long w = 0;
    for (int t = 0; t < 5; t++)
        for (int q = 0; q < 4; q++) w |= (unsigned long long)tet_node(t0 + t, q) << (t * 12 + q * 3);
    return w;
}
__device__ __forceinline__ int tet_node_rt(int t, int q) {
    constexpr unsigned long long lo = pack_tets(0), hi = pack_tets(5);
    unsigned long long w = t < 5 ? lo : hi;
    int sh = (t < 5 ? t : t - 5) * 12 + q * 3;
    return (int)((w >> sh) & 7ull);
}

// One phase on the device.  The transcendental values of a softening table
// whose angles do not vary are evaluated once on the host with the host C
// library (the reference's libm), so that a constant-angle Mohr-Coulomb run
// rounds like the reference.
struct DevMaterial {
    double density, alpha, beta, lambda, mu;
    int nsegments, yield_mc;
    double plstrain[SNAC_MAX_SEGMENTS + 1];
    double fric[SNAC_MAX_SEGMENTS + 1];
    double dil[SNAC_MAX_SEGMENTS + 1];
    double coh[SNAC_MAX_SEGMENTS + 1];
    double ten_off;
    double vis_min, vis_max, refvisc, refsrate, reftemp, H, srexponent;
    double thermal_conduct, heat_capacity;
    // constant factors of the Arrhenius viscosity, evaluated on the host with
    // the same IEEE operations: 1/srexponent - 1, H/R, 1/(reftemp + 273.15), RN(1/refsrate)
    double vp_expo, vp_hr, vp_irt, vp_zrs;
    // host-evaluated per-segment 1/(plstrain[i+1] - plstrain[i]) and, for a
    // constant angle, (1 + sin)/(1 - sin) of friction and dilation,
    // sqrt of the former and RN(1 / tan(friction))
    double zpl[SNAC_MAX_SEGMENTS];
    double anphi0, anpsi0, sq_anphi0, ztan_fric0;
    // host-evaluated transcendentals (valid when the *_const flag is set)
    int fric_const, dil_const;
    double fric0, sin_fric0, tan_fric0;
    double dil0, sin_dil0, tan_dil0;
    // Drucker-Prager phase (yield_mc == 0, visco-plastic hook): maxiterations, constitutivetolerance
    int dp_maxit;
    double dp_tol;
};

// Device-resident scalars of one model (everything a captured step reads).
struct DevScalars {
    double dt;
    double dt_rot;                   // dt of the element update still to apply (fused pipeline)
    double speed_of_sound;
    double min_length_scale;
    double vmax;
    double init_min_length_scale;
    unsigned long long minls_bits;   // running min of |V/A| (non-negative doubles order as integers)
    unsigned long long vmax_bits;    // running max of |v| over velocity-BC nodes
    long long time_step;
    double current_time;             // AbstractContext currentTime: the sum of the steps' dt
    double topo_grad_max;            // Snac_Context topoGradMax: running max of |grad y| on the top surface
    int pos_parity;                  // which of the two coordinate buffers is current
    int want_scalars;                // the next step stores the element scalars (a dump follows it)
    int status;                      // first error (SNAC_GPU_E*), 0 if none
    long long err_index;
    long long launches;
    double inertial_density0;        // (lambda + 2 mu) / c^2 of phase 0 at the current speed of sound c (dynamic dt)
    unsigned blocks_done;            // blocks of k_min_length_scale_sync finished (0 between launches)
    unsigned pad;
    // k_heat_flux_min_length_scale's per-block minima, spread over 32
    // addresses (+inf between steps)
    unsigned long long minls_slot[32];
};

__device__ __forceinline__ void report(DevScalars* sc, int code, long long index) {
    if (atomicCAS(&sc->status, 0, code) == 0) sc->err_index = index;
}

#ifndef SNAC_MARKSTEIN_DIV
#define SNAC_MARKSTEIN_DIV 2
#endif

// ---- correctly rounded division by a known reciprocal --------------------------------
// With z = RN(1/y) (the correctly rounded reciprocal) and q0 = RN(x z),
// which is within one ulp of x / y, the remainder r = x - q0 y is exact in
// one FMA and RN(q0 + r z) is the correctly rounded quotient RN(x / y):
// Markstein's theorem (P. Markstein, "Computation of elementary functions on
// the IBM RISC System/6000 processor", IBM J. Res. Dev. 34(1), 1990; J.-M.
// Muller et al., Handbook of Floating-Point Arithmetic, 2nd ed., 2018,
// ch. 4).  So a division by a constant (z a literal) or several divisions by
// one divisor (z computed once) cost a multiply and two FMAs each instead of
// a full division.  The theorem needs the quotient and divisor in the normal
// range without overflow or underflow: operands outside a safe exponent
// window and negative divisors (checked with integer operations on the high
// and low words) take the IEEE division; zeros get their sign from the form
// of the correction step (markstein() below).  SNAC_MARKSTEIN_DIV = 1
// uses it for the constant divisors only, 2 also for shared divisors.  The device self-test
// (snac_gpu_selftest_division) compares every helper with the hardware '/'
// on random operands, near-ties included.

// RN(1/y)
__host__ __device__ __forceinline__ double recip(double y) {
#ifdef __CUDA_ARCH__
    return __drcp_rn(y);
#else
    return 1.0 / y;
#endif
}

// biased exponent of x (0 for zeros and subnormals, 2047 for Inf/NaN)
__host__ __device__ __forceinline__ unsigned biased_exp(double x) {
    unsigned long long b;
    memcpy(&b, &x, 8);
    return (unsigned)(b >> 52) & 0x7ffu;
}
// |x| in [2^lo, 2^(hi+1)) by integer tests (keeps the checks off the FP64 pipe)
template <int LO, int HI>
__host__ __device__ __forceinline__ bool exp_within(double x) {
    return biased_exp(x) - (unsigned)(1023 + LO) <= (unsigned)(HI - LO);
}
__host__ __device__ __forceinline__ void hi_lo(double x, unsigned& h, unsigned& l) {
#ifdef __CUDA_ARCH__
    h = (unsigned)__double2hiint(x);
    l = (unsigned)__double2loint(x);
#else
    unsigned long long b;
    memcpy(&b, &x, 8);
    h = (unsigned)(b >> 32);
    l = (unsigned)b;
#endif
}
// x = +-0 or |x| in [2^lo, 2^(hi+1)), on the high and low words: the sign
// is shifted out of the high word and the window is one unsigned compare
template <int LO, int HI>
__host__ __device__ __forceinline__ bool zero_or_within(double x) {
    unsigned h, l;
    hi_lo(x, h, l);
    const bool win = (h << 1) - ((unsigned)(1023 + LO) << 21) <= ((unsigned)(HI - LO + 1) << 21) - 1u;
    return win | (((h & 0x7fffffffu) | l) == 0u);
}
// y in [2^lo, 2^(hi+1)) and positive (a set sign bit puts the high word
// above the window)
template <int LO, int HI>
__host__ __device__ __forceinline__ bool positive_within(double y) {
    unsigned h, l;
    hi_lo(y, h, l);
    return h - ((unsigned)(1023 + LO) << 20) <= ((unsigned)(HI - LO + 1) << 20) - 1u;
}

// The IEEE division for the rare operands outside the window, as a call: its
// code (with its own special-case paths) then is not inlined at each of the
// few dozen division sites of an element kernel, where it cost registers and
// instruction scheduling on the common path.
__host__ __device__ __noinline__ double ieee_div(double x, double y) { return x / y; }

// The correction step RN(q0 + r z), r = x - q0 y, written as
// -RN(-r z - q0): the same value (round-to-nearest is symmetric), and for
// y > 0 a zero x also gets the IEEE quotient's sign (+-0 / y = +-0), which
// RN(q0 + r z) gives -0 / y as +0.  So zeros need no test of their own.
__host__ __device__ __forceinline__ double markstein(double x, double y, double z, double q0) {
    const double r = fma(-q0, y, x);
    return -fma(-r, z, -q0);
}

// RN(x / c) for a constant c with z = RN(1/c) and 1 <= c <= 16
__host__ __device__ __forceinline__ double dvk(double x, double c, double z) {
#if SNAC_MARKSTEIN_DIV >= 1
    const double q0 = x * z;
    const double q = markstein(x, c, z, q0);
    if (!zero_or_within<-900, 900>(x)) return ieee_div(x, c);
    return q;
#else
    (void)z;
    return x / c;
#endif
}

// RN(x / y) given z = RN(1/y)
__host__ __device__ __forceinline__ double dvz(double x, double y, double z) {
#if SNAC_MARKSTEIN_DIV >= 2
    const double q0 = x * z;
    const double q = markstein(x, y, z, q0);
    if (!(zero_or_within<-450, 450>(x) && positive_within<-450, 450>(y))) return ieee_div(x, y);
    return q;
#else
    (void)z;
    return x / y;
#endif
}

// Groups of quotients, in place: one window test and one branch for the
// group instead of one per quotient (a branch per division splits the
// instruction schedule); a group with any operand outside the window takes
// the IEEE division for all of its members.
template <int N>
__host__ __device__ __forceinline__ void dvk_n(double (&x)[N], double c, double z) {
#if defined(__CUDA_ARCH__) && SNAC_MARKSTEIN_DIV >= 1
    double q[N];
    bool ok = true;
#pragma unroll
    for (int i = 0; i < N; i++) {
        q[i] = markstein(x[i], c, z, x[i] * z);
        ok = ok & zero_or_within<-900, 900>(x[i]);
    }
    if (ok) {
#pragma unroll
        for (int i = 0; i < N; i++) x[i] = q[i];
    } else {
#pragma unroll
        for (int i = 0; i < N; i++) x[i] = ieee_div(x[i], c);
    }
#else
    (void)z;
    for (int i = 0; i < N; i++) x[i] = x[i] / c;
#endif
}
template <int N>
__host__ __device__ __forceinline__ void dvz_n(double (&x)[N], double y, double z) {
#if defined(__CUDA_ARCH__) && SNAC_MARKSTEIN_DIV >= 2
    double q[N];
    bool ok = positive_within<-450, 450>(y);
#pragma unroll
    for (int i = 0; i < N; i++) {
        q[i] = markstein(x[i], y, z, x[i] * z);
        ok = ok & zero_or_within<-450, 450>(x[i]);
    }
    if (ok) {
#pragma unroll
        for (int i = 0; i < N; i++) x[i] = q[i];
    } else {
#pragma unroll
        for (int i = 0; i < N; i++) x[i] = ieee_div(x[i], y);
    }
#else
    (void)z;
    for (int i = 0; i < N; i++) x[i] = x[i] / y;
#endif
}
constexpr double Z3 = 0x1.5555555555555p-2, Z6 = 0x1.5555555555555p-3;  // RN(1/3), RN(1/6)

__host__ __device__ __forceinline__ double dv(double x, double y) { return x / y; }
// division by the constants the reference uses; the reciprocal is RN(1/c)
__host__ __device__ __forceinline__ double dv3(double x) { return dvk(x, 3.0, 0x1.5555555555555p-2); }
__host__ __device__ __forceinline__ double dv6(double x) { return dvk(x, 6.0, 0x1.5555555555555p-3); }
__host__ __device__ __forceinline__ double dv9(double x) { return dvk(x, 9.0, 0x1.c71c71c71c71cp-4); }
__host__ __device__ __forceinline__ double dv10(double x) { return dvk(x, 10.0, 0x1.999999999999ap-4); }

struct V3 {
    double x, y, z;
};

// ---- Tetrahedra.c:44-113 ------------------------------------------------------------
__device__ __forceinline__ double tet_volume(const V3& c1, const V3& c2, const V3& c3, const V3& c4) {
    double x2 = c2.x - c1.x, y2 = c2.y - c1.y, z2 = c2.z - c1.z;
    double x3 = c3.x - c1.x, y3 = c3.y - c1.y, z3 = c3.z - c1.z;
    double x4 = c4.x - c1.x, y4 = c4.y - c1.y, z4 = c4.z - c1.z;
    double v = dv6(x4 * (y2 * z3 - z2 * y3) + y4 * (z2 * x3 - x2 * z3) + z4 * (x2 * y3 - x3 * y2));
    return fabs(v);
}

// Tetrahedra_SurfaceArea and Tetrahedra_SurfaceNormal evaluate the same cross
// product and the same square root; computing it once gives the same bits.
__device__ __forceinline__ void tet_face(const V3& c1, const V3& c2, const V3& c3, double& area, V3& n) {
    double x2 = c2.x - c1.x, y2 = c2.y - c1.y, z2 = c2.z - c1.z;
    double x3 = c3.x - c1.x, y3 = c3.y - c1.y, z3 = c3.z - c1.z;
    double a = y2 * z3 - z2 * y3;
    double b = z2 * x3 - x2 * z3;
    double c = x2 * y3 - y2 * x3;
    double s = sqrt(a * a + b * b + c * c);
    area = s * 0.5;  // a product with 2^-k rounds exactly as the quotient by 2^k
    double t[3] = {a, b, c};
    dvz_n(t, s, recip(s));
    n = {t[0], t[1], t[2]};
}

struct TetGeom {
    double V;
    double zV;  // RN(1/V), shared by every division by V
    double A[4];
    V3 n[4];
};

__device__ __forceinline__ void tet_geometry(const V3 c[4], TetGeom& g) {
    g.V = tet_volume(c[0], c[1], c[2], c[3]);
    g.zV = recip(g.V);
#pragma unroll
    for (int f = 0; f < 4; f++)
        tet_face(c[face_node(f, 0)], c[face_node(f, 1)], c[face_node(f, 2)], g.A[f], g.n[f]);
}

__device__ __forceinline__ double comp(const V3& v, int d) { return d == 0 ? v.x : (d == 1 ? v.y : v.z); }

// sum_k w_k,a * n_face(k),b * A_face(k) over the tet's nodes k (node k pairs
// with face (1,2,3,0)[k]), StrainRate.c:65-184 / UpdateElement.c:145-219
__device__ __forceinline__ double face_sum(const V3 w[4], int a, const TetGeom& g, int b) {
    return comp(w[0], a) * comp(g.n[1], b) * g.A[1] + comp(w[1], a) * comp(g.n[2], b) * g.A[2] +
           comp(w[2], a) * comp(g.n[3], b) * g.A[3] + comp(w[3], a) * comp(g.n[0], b) * g.A[0];
}

// The reference writes the spin and shear sums as one left-to-right chain
// a0+a1+a2+a3 -/+ b0 -/+ b1 -/+ b2 -/+ b3 (UpdateElement.c:145-219,
// StrainRate.c:101-184); these keep that chain.
__device__ __forceinline__ double spin_sum(const V3 v[4], const TetGeom& g, int a, int b) {
    return comp(v[0], a) * comp(g.n[1], b) * g.A[1] + comp(v[1], a) * comp(g.n[2], b) * g.A[2] +
           comp(v[2], a) * comp(g.n[3], b) * g.A[3] + comp(v[3], a) * comp(g.n[0], b) * g.A[0] -
           comp(v[0], b) * comp(g.n[1], a) * g.A[1] - comp(v[1], b) * comp(g.n[2], a) * g.A[2] -
           comp(v[2], b) * comp(g.n[3], a) * g.A[3] - comp(v[3], b) * comp(g.n[0], a) * g.A[0];
}
__device__ __forceinline__ double shear_sum(const V3 v[4], const TetGeom& g, int a, int b) {
    return comp(v[0], a) * comp(g.n[1], b) * g.A[1] + comp(v[1], a) * comp(g.n[2], b) * g.A[2] +
           comp(v[2], a) * comp(g.n[3], b) * g.A[3] + comp(v[3], a) * comp(g.n[0], b) * g.A[0] +
           comp(v[0], b) * comp(g.n[1], a) * g.A[1] + comp(v[1], b) * comp(g.n[2], a) * g.A[2] +
           comp(v[2], b) * comp(g.n[3], a) * g.A[3] + comp(v[3], b) * comp(g.n[0], a) * g.A[0];
}

// StrainRate.c:65-184, before the mixed-discretisation correction;
// sr = (xx, yy, zz, xy, xz, yz)
__device__ __forceinline__ void tet_strain_rate(const V3 v[4], const TetGeom& g, double sr[6]) {
    double t[6] = {-1.0f * (face_sum(v, 0, g, 0)), -1.0f * (face_sum(v, 1, g, 1)), -1.0f * (face_sum(v, 2, g, 2)),
                   -0.5f * (shear_sum(v, g, 0, 1)), -0.5f * (shear_sum(v, g, 0, 2)), -0.5f * (shear_sum(v, g, 1, 2))};
    dvk_n(t, 3.0, Z3);
    dvz_n(t, g.V, g.zV);
#pragma unroll
    for (int a = 0; a < 6; a++) sr[a] = t[a];
}

// spin rates r01, r02, r12 of a tet, UpdateElement.c:145-219
__device__ __forceinline__ void spin_rates(const V3 v[4], const TetGeom& g, double (&r)[3]) {
    // RN(0.5 / V) = 0.5 RN(1 / V) exactly while 1 / V is a normal number
    const double hV = exp_within<-1000, 1000>(g.V) ? 0.5 * g.zV : ieee_div(0.5, g.V);
    r[0] = -(hV) * (spin_sum(v, g, 0, 1));
    r[1] = -(hV) * (spin_sum(v, g, 0, 2));
    r[2] = -(hV) * (spin_sum(v, g, 1, 2));
    dvk_n(r, 3.0, Z3);
}

// The spin rates (UpdateElement.c:145-219) and the strain rate
// (StrainRate.c:65-184) of one tet from the same velocities and geometry,
// as the fused element kernel needs both: the chains
// a0+a1+a2+a3 -/+ b0 -/+ b1 -/+ b2 -/+ b3 of a spin sum and of the matching
// shear sum share their products and their prefix a0+..+a3, which are
// formed once here; every result has the bits of spin_rates and
// tet_strain_rate.
__device__ __forceinline__ void spin_and_strain_rates(const V3 v[4], const TetGeom& g, double (&r)[3], double sr[6]) {
    double t[6];
    t[0] = -1.0f * (face_sum(v, 0, g, 0));
    t[1] = -1.0f * (face_sum(v, 1, g, 1));
    t[2] = -1.0f * (face_sum(v, 2, g, 2));
    constexpr int PA[3] = {0, 0, 1}, PB[3] = {1, 2, 2};
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const int a = PA[k], b = PB[k];
        const double pre = comp(v[0], a) * comp(g.n[1], b) * g.A[1] + comp(v[1], a) * comp(g.n[2], b) * g.A[2] +
                           comp(v[2], a) * comp(g.n[3], b) * g.A[3] + comp(v[3], a) * comp(g.n[0], b) * g.A[0];
        const double q0 = comp(v[0], b) * comp(g.n[1], a) * g.A[1], q1 = comp(v[1], b) * comp(g.n[2], a) * g.A[2],
                     q2 = comp(v[2], b) * comp(g.n[3], a) * g.A[3], q3 = comp(v[3], b) * comp(g.n[0], a) * g.A[0];
        r[k] = pre - q0 - q1 - q2 - q3;
        t[3 + k] = -0.5f * (pre + q0 + q1 + q2 + q3);
    }
    const double hV = exp_within<-1000, 1000>(g.V) ? 0.5 * g.zV : ieee_div(0.5, g.V);
#pragma unroll
    for (int k = 0; k < 3; k++) r[k] = -(hV) * (r[k]);
    dvk_n(r, 3.0, Z3);
    dvk_n(t, 3.0, Z3);
    dvz_n(t, g.V, g.zV);
#pragma unroll
    for (int a = 0; a < 6; a++) sr[a] = t[a];
}

// Jaumann rotation of the stress with the spin rates r, UpdateElement.c:145-265
// (the strain is zeroed first, :81, so its own rotation leaves it zero); s01
// takes "+ r12*s02".
__device__ __forceinline__ void rotate_stress_by(const double (&r)[3], double dt, double s[6]) {
    const double r01 = r[0], r02 = r[1], r12 = r[2];
    s[0] += (2.0f * r01 * s[3] + 2.0f * r02 * s[4]) * dt;
    s[1] += (2.0f * (-1.0f * r01) * s[3] + 2.0f * r12 * s[5]) * dt;
    s[2] += (2.0f * (-1.0f * r02) * s[4] + 2.0f * (-1.0f * r12) * s[5]) * dt;
    s[3] += (r01 * (s[1] - s[0])) * dt + (r02 * s[5] + r12 * s[4]) * dt;
    s[4] += (r02 * (s[2] - s[0])) * dt + (r01 * s[5] - r12 * s[3]) * dt;
    s[5] += (r12 * (s[2] - s[1])) * dt + ((-1.0f * r01) * s[4] - r02 * s[3]) * dt;
}

// Jaumann rotation of the stress, UpdateElement.c:145-265 (the strain is
// zeroed first, :81, so its own rotation leaves it zero); s01 takes "+ r12*s02".
__device__ __forceinline__ void rotate_stress(const V3 v[4], const TetGeom& g, double dt, double s[6]) {
    // RN(0.5 / V) = 0.5 RN(1 / V) exactly while 1 / V is a normal number
    double r[3];
    spin_rates(v, g, r);
    const double r01 = r[0], r02 = r[1], r12 = r[2];
    s[0] += (2.0f * r01 * s[3] + 2.0f * r02 * s[4]) * dt;
    s[1] += (2.0f * (-1.0f * r01) * s[3] + 2.0f * r12 * s[5]) * dt;
    s[2] += (2.0f * (-1.0f * r02) * s[4] + 2.0f * (-1.0f * r12) * s[5]) * dt;
    s[3] += (r01 * (s[1] - s[0])) * dt + (r02 * s[5] + r12 * s[4]) * dt;
    s[4] += (r02 * (s[2] - s[0])) * dt + (r01 * s[5] - r12 * s[3]) * dt;
    s[5] += (r12 * (s[2] - s[1])) * dt + ((-1.0f * r01) * s[4] - r02 * s[3]) * dt;
}

// ---- plastic/Constitutive.c:249-410: cyclic Jacobi (Numerical Recipes
// jacobi/eigsrt) on the symmetric stress, then principal values ascending
// (most compressive first) and their directions cn[k] = eigenvector k.
// The three (ip,iq) pairs and their rotate loops are spelled out so that the
// whole solver lives in registers.
__host__ __device__ __forceinline__ void jrot(double& aij, double& akl, double s, double tau) {
    double g = aij, h = akl;
    aij = g - s * (h + g * tau);
    akl = h + s * (g - h * tau);
}

struct Jac {
    double a01, a02, a12;  // off-diagonal part (the diagonal lives in d/b)
    double d[3], b[3], z[3];
    double v[3][3];
};

template <int IP, int IQ>
__host__ __device__ __forceinline__ void jac_pair(Jac& J, int i, double tresh) {
    double& apq = (IP == 0 && IQ == 1) ? J.a01 : (IP == 0 && IQ == 2) ? J.a02 : J.a12;
    double g = 100.0f * fabs(apq);
    if ((i > 4) && (double)(fabs(J.d[IP]) + g) == (double)fabs(J.d[IP]) &&
        (double)(fabs(J.d[IQ]) + g) == (double)fabs(J.d[IQ])) {
        apq = 0.0f;
    } else if (fabs(apq) > tresh) {
        double h = J.d[IQ] - J.d[IP], t;
        if ((fabs(h) + g) == fabs(h)) {
            t = dv(apq, h);
        } else {
            double theta = dv(0.5f * h, apq);
            t = dv(1.0f, fabs(theta) + sqrt(1.0f + theta * theta));
            if (theta < 0.0f) t *= -1.0f;
        }
        double c = dv(1.0f, sqrt(1.0f + t * t));
        double s = t * c;
        double tau = dv(s, 1.0f + c);
        h = t * apq;
        J.z[IP] -= h;
        J.z[IQ] += h;
        J.d[IP] -= h;
        J.d[IQ] += h;
        apq = 0.0f;
        // the reference's three rotate loops for this pair (j < ip, ip < j < iq, j > iq)
        if (IP == 0 && IQ == 1) jrot(J.a02, J.a12, s, tau);          // j = 2 > iq
        if (IP == 0 && IQ == 2) jrot(J.a01, J.a12, s, tau);          // j = 1 between
        if (IP == 1 && IQ == 2) jrot(J.a01, J.a02, s, tau);          // j = 0 < ip
#pragma unroll
        for (int j = 0; j < 3; j++) jrot(J.v[j][IP], J.v[j][IQ], s, tau);
    }
}

__host__ __device__ void principal_stresses(const double st[6], double sp[3], double cn[3][3]) {
    Jac J;
    J.a01 = st[3];
    J.a02 = st[4];
    J.a12 = st[5];
#pragma unroll
    for (int ip = 0; ip < 3; ip++) {
#pragma unroll
        for (int iq = 0; iq < 3; iq++) J.v[ip][iq] = 0.0f;
        J.v[ip][ip] = 1.0f;
    }
#pragma unroll
    for (int ip = 0; ip < 3; ip++) {
        J.b[ip] = J.d[ip] = st[ip];
        J.z[ip] = 0.0f;
    }
    for (int i = 1; i <= 50; i++) {
        double sm = 0.0f;
        sm += fabs(J.a01);
        sm += fabs(J.a02);
        sm += fabs(J.a12);
        if (sm == 0.0f) break;
        double tresh = (i < 4) ? dv9(0.2f * sm) : 0.0f;
        jac_pair<0, 1>(J, i, tresh);
        jac_pair<0, 2>(J, i, tresh);
        jac_pair<1, 2>(J, i, tresh);
#pragma unroll
        for (int ip = 0; ip < 3; ip++) {
            J.b[ip] += J.z[ip];
            J.d[ip] = J.b[ip];
            J.z[ip] = 0.0f;
        }
    }
    double d[3] = {J.d[0] * -1.0f, J.d[1] * -1.0f, J.d[2] * -1.0f};
    // eigsrt: descending, ">=" keeps the later index on ties
#pragma unroll
    for (int i = 0; i < 2; i++) {
        int k = i;
        double p = d[i];
#pragma unroll
        for (int j = i + 1; j < 3; j++)
            if (d[j] >= p) {
                k = j;
                p = d[j];
            }
        if (k != i) {
            // swap entry i with entry k (k > i), columns of v likewise
#pragma unroll
            for (int kk = i + 1; kk < 3; kk++)
                if (kk == k) {
                    d[kk] = d[i];
                    d[i] = p;
#pragma unroll
                    for (int j = 0; j < 3; j++) {
                        double q = J.v[j][i];
                        J.v[j][i] = J.v[j][kk];
                        J.v[j][kk] = q;
                    }
                }
        }
    }
#pragma unroll
    for (int i = 0; i < 3; i++) {
        sp[i] = d[i] * -1.0f;
#pragma unroll
        for (int j = 0; j < 3; j++) cn[i][j] = J.v[j][i];
    }
}

// True when the tet provably does not reach the Mohr-Coulomb or tension
// surface, so the reference would leave its trial stress untouched: the
// exact eigenvalues lie in the Gershgorin interval [lo, hi], the Jacobi
// values are within ~1e-15 of the stress scale of them, and the margin asked
// for is 1e-9 of that scale.  Skipping the eigen-solve then changes no bit.
__host__ __device__ __forceinline__ bool surely_elastic(const double st[6], double cohesion, double anphi,
                                                       double sqrt_anphi, double stc) {
    double r0 = fabs(st[3]) + fabs(st[4]);
    double r1 = fabs(st[3]) + fabs(st[5]);
    double r2 = fabs(st[4]) + fabs(st[5]);
    double hi = fmax(st[0] + r0, fmax(st[1] + r1, st[2] + r2));
    double lo = fmin(st[0] - r0, fmin(st[1] - r1, st[2] - r2));
    double scale = fabs(st[0]) + fabs(st[1]) + fabs(st[2]) + 2.0 * (r0 + r1 + r2);
    double cterm = 2.0 * cohesion * sqrt_anphi;
    double tol_t = 1e-9 * (scale + fabs(stc)) + 1e-300;
    double tol_s = 1e-9 * (scale * (1.0 + anphi) + fabs(cterm)) + 1e-300;
    bool no_tension = hi - stc < -tol_t;
    bool no_shear = (lo - hi * anphi + cterm) > tol_s;
    return no_tension && no_shear && anphi > 0.0;
}

// PI/180 with PI = M_PI, plastic/Constitutive.c:44-55
__device__ __forceinline__ double degrad() { return 3.14159265358979323846 / 180.0f; }

__device__ __forceinline__ double sin_fric(const DevMaterial& m, double phi) {
    return (m.fric_const && phi == m.fric0) ? m.sin_fric0 : sin(phi * degrad());
}
__device__ __forceinline__ double tan_fric(const DevMaterial& m, double phi) {
    return (m.fric_const && phi == m.fric0) ? m.tan_fric0 : tan(phi * degrad());
}
__device__ __forceinline__ double sin_dil(const DevMaterial& m, double psi) {
    return (m.dil_const && psi == m.dil0) ? m.sin_dil0 : sin(psi * degrad());
}
__device__ __forceinline__ double tan_dil(const DevMaterial& m, double psi) {
    return (m.dil_const && psi == m.dil0) ? m.tan_dil0 : tan(psi * degrad());
}

// viscoplastic/Constitutive.c:372-518, the Drucker-Prager return map of one
// tet after its viscous update.  s: the stress (xx, yy, zz, xy, xz, yz); sd:
// the updated deviatoric diagonal; S0: the stress before the viscous update;
// e: the strain increment; pst: the accumulated plastic strain tensor.  Up
// to mite passes: shear (h > 0) or tension increments; with more than one
// pass the viscous update is redone with them and the yield functions
// evaluated again until both are below tol times their larger first value.
// The increments accumulate in pst, whose second invariant becomes eps_p.
// palam, the previous pass's multiplier for a pass whose own is negative,
// is an uninitialised function-scope variable in the reference on its first
// use; here it starts at 0.  IEEE division and square root throughout (a
// rarely taken path).  Returns whether the tet yielded.
__device__ __noinline__ bool dp_return_map(double s[6], double sd[3], const double S0[6], const double e[6],
                                           double vic1, double vic2, double rmu, double bulkm, double qphi,
                                           double qpsi, double kphi, double st, double tol, int mite, double pst[6],
                                           double& eps_p) {
    double I1 = (s[0] + s[1] + s[2]) / 3.;
    double J2 = sqrt(0.5 * (sd[0] * sd[0] + sd[1] * sd[1] + sd[2] * sd[2]) + s[3] * s[3] + s[4] * s[4] + s[5] * s[5]);
    double fs = J2 + I1 * qphi - kphi;
    double ft = I1 - st;
    if (!(fs > 0.0f || ft > 0.0f)) return false;
    double dep[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0}, depm;
    const double tolerf = fs > ft ? tol * fs : tol * ft;
    double previousfs = fs, previousft = ft, palam = 0.0, alam;
    for (int ite = 0; ite < mite; ite++) {
        const double aP = sqrt(1.0f + qphi * qphi) - qphi;
        const double sP = kphi - qphi * st;
        const double h = J2 - sP - aP * (I1 - st);
        if (h > 0.0f) {  // shear
            alam = fs / (bulkm * qphi * qpsi + rmu);
            if (alam < 0.0) alam = palam * (previousfs / (previousfs - fs));
            for (int a = 0; a < 3; a++) dep[a] = alam * (0.5 * sd[a] / J2 + qpsi / 3.);
            for (int a = 3; a < 6; a++) dep[a] = alam * 0.5 * (s[a]) / J2;
        } else {  // tension (the shear increments of a previous pass stay)
            alam = ft / bulkm;
            if (alam < 0.0) alam = palam * (previousft / (previousfs - ft));
            for (int a = 0; a < 3; a++) dep[a] = alam / 3.;
        }
        if (mite == 1) break;
        depm = (dep[0] + dep[1] + dep[2]) / 3.0f;
        const double trace_strain = e[0] + e[1] + e[2];
        double strd[3];
        for (int a = 0; a < 3; a++) strd[a] = e[a] - dep[a] - (trace_strain) / 3.0f + depm;
        const double trace_stress = S0[0] + S0[1] + S0[2];
        for (int a = 0; a < 3; a++) sd[a] = S0[a] - trace_stress / 3.;
        for (int a = 0; a < 3; a++) sd[a] = (sd[a] * vic1 + 2.0f * rmu * strd[a]) * vic2;
        for (int a = 3; a < 6; a++) s[a] = (S0[a] * vic1 + 2.0f * rmu * (e[a] - dep[a])) * vic2;
        const double VolumicStress = trace_stress / 3.0f + bulkm * (trace_strain - 3. * depm);
        for (int a = 0; a < 3; a++) s[a] = sd[a] + VolumicStress;
        I1 = (s[0] + s[1] + s[2]) / 3.;
        for (int a = 0; a < 3; a++) sd[a] = s[a] - I1;
        J2 = sqrt(0.5 * (sd[0] * sd[0] + sd[1] * sd[1] + sd[2] * sd[2]) + s[3] * s[3] + s[4] * s[4] + s[5] * s[5]);
        previousfs = fs;
        previousft = ft;
        palam = alam;
        fs = J2 + I1 * qphi - kphi;
        ft = I1 - st;
        if (fs < tolerf && ft < tolerf) break;
    }
    for (int a = 0; a < 6; a++) pst[a] += dep[a];
    depm = (pst[0] + pst[1] + pst[2]) / 3.0f;
    eps_p = sqrt(0.5f * ((pst[0] - depm) * (pst[0] - depm) + (pst[1] - depm) * (pst[1] - depm) +
                         (pst[2] - depm) * (pst[2] - depm)) +
                 pst[3] * pst[3] + pst[4] * pst[4] + pst[5] * pst[5]);
    return true;
}

// Mohr-Coulomb composite yield + return map in principal space, shared by
// plastic/Constitutive.c:180-237 and viscoplastic/Constitutive.c:305-370.
// Returns 1 when the tet yielded (stress resolved back, plastic strain grown).
__device__ __forceinline__ int mc_return_map(double sp[3], const double cn[3][3], double st6[6], double& eps_p,
                                             double cohesion, double hardening, double anphi, double anpsi,
                                             double st, double a1, double a2) {
    double alam, dep1, dep2, dep3, depm;
    double fs = sp[0] - sp[2] * anphi + 2 * cohesion * sqrt(anphi);
    double ft = sp[2] - st;
    if (!(fs < 0.0f || ft > 0.0f)) return 0;
    double aP = sqrt(1.0f + anphi * anphi) + anphi;
    double sP = st * anphi - 2 * cohesion * sqrt(anphi);
    double h = sp[2] - st + aP * (sp[0] - sP);
    if (h < 0.0f) {
        alam = dv(fs, a1 - a2 * anpsi + a1 * anphi * anpsi - a2 * anphi + 2.0 * sqrt(anphi) * hardening);
        sp[0] -= alam * (a1 - a2 * anpsi);
        sp[1] -= alam * a2 * (1.0f - anpsi);
        sp[2] -= alam * (a2 - a1 * anpsi);
        dep1 = alam;
        dep2 = 0.0f;
        dep3 = -alam * anpsi;
    } else {
        alam = dv(ft, a1);
        sp[0] -= alam * a2;
        sp[1] -= alam * a2;
        sp[2] -= alam * a1;
        dep1 = 0.0f;
        dep2 = 0.0f;
        dep3 = alam;
    }
    depm = dv3(dep1 + dep2 + dep3);
    eps_p += sqrt(0.5f * ((dep1 - depm) * (dep1 - depm) + (dep2 - depm) * (dep2 - depm) +
                          (dep3 - depm) * (dep3 - depm) + depm * depm));
    double r[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int m = 0; m < 3; m++)
        for (int n = m; n < 3; n++)
            for (int k = 0; k < 3; k++) r[m][n] += cn[k][m] * cn[k][n] * sp[k];
    st6[0] = r[0][0];
    st6[1] = r[1][1];
    st6[2] = r[2][2];
    st6[3] = r[0][1];
    st6[4] = r[0][2];
    st6[5] = r[1][2];
    return 1;
}

// Power-law / Arrhenius viscosity, viscoplastic/Constitutive.c:186-210 and
// maxwell/Constitutive.c:122-142, clipped to [vis_min, vis_max].
// The unclipped viscosity refvisc (srJ2/refsrate)^expo exp(H/R (1/T - 1/Tref)),
// evaluated as one exponential, refvisc exp(expo ln(srJ2/refsrate) +
// H/R (1/T - 1/Tref)): the same value to a few ulp (the exponent is O(10)),
// one transcendental instead of pow and exp.  The reference's libm pow/exp
// are not reproduced bit for bit on the device either way, so visco-plastic
// and Maxwell runs are compared with the oracle at a tolerance.
__device__ __forceinline__ double arrhenius_base(const DevMaterial& M, double refvisc, double srJ2, double avgTemp) {
    return refvisc * exp(M.vp_expo * log(dvz(srJ2, M.refsrate, M.vp_zrs)) +
                         M.vp_hr * (recip(avgTemp + 273.15) - M.vp_irt));
}

__device__ __forceinline__ double arrhenius_viscosity(const DevMaterial& M, double refvisc, double srJ2,
                                                      double avgTemp) {
    double eta = arrhenius_base(M, refvisc, srJ2, avgTemp);
    if (eta < M.vis_min) eta = M.vis_min;
    if (eta > M.vis_max) eta = M.vis_max;
    return eta;
}

// Maxwell visco-elastic update of one tet, viscoplastic/Constitutive.c:211-257
// and maxwell/Constitutive.c:146-183 (identical arithmetic).
__device__ __forceinline__ void maxwell_update(double s[6], const double e[6], double stressd[3],
                                               const double straind[3], double trace_stress3, double trace_strain,
                                               double rmu, double eta, double dt, double bulkm, double& vic1,
                                               double& vic2) {
    double temp = dv(rmu, 2.0f * (eta)) * dt;
    vic1 = 1.0f - temp;
    vic2 = recip(1.0f + temp);  // RN(1 / x), the same bits as 1.0 / x
    stressd[0] = (stressd[0] * vic1 + 2.0f * rmu * straind[0]) * vic2;
    stressd[1] = (stressd[1] * vic1 + 2.0f * rmu * straind[1]) * vic2;
    stressd[2] = (stressd[2] * vic1 + 2.0f * rmu * straind[2]) * vic2;
    s[3] = (s[3] * vic1 + 2.0f * rmu * e[3]) * vic2;
    s[4] = (s[4] * vic1 + 2.0f * rmu * e[4]) * vic2;
    s[5] = (s[5] * vic1 + 2.0f * rmu * e[5]) * vic2;
    double VolumicStress = trace_stress3 + bulkm * trace_strain;
    s[0] = stressd[0] + VolumicStress;
    s[1] = stressd[1] + VolumicStress;
    s[2] = stressd[2] + VolumicStress;
}
__device__ __forceinline__ void maxwell_update(double s[6], const double e[6], double stressd[3],
                                               const double straind[3], double trace_stress3, double trace_strain,
                                               double rmu, double eta, double dt, double bulkm) {
    double vic1, vic2;
    maxwell_update(s, e, stressd, straind, trace_stress3, trace_strain, rmu, eta, dt, bulkm, vic1, vic2);
}

}  // namespace snac
