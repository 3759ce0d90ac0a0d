/*
 * snac_oracle.c — CPU restatement of SNAC's explicit Lagrangian step.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, never the product): see
 * snac_oracle.h.  Every function cites the reference file:line it restates;
 * paths are relative to the SNAC source tree.  Arithmetic is written in the
 * reference's evaluation order, in double precision, and must be compiled
 * without FMA contraction (-ffp-contract=off) so that it rounds like the
 * reference's x86-64 -O3 build.
 *
 * Float literals of the reference (0.45f, 3.0e-11f, 1.0e+27f, 0.2f, ...) are
 * kept as float literals here: C promotes them to double exactly as the
 * reference does.
 */
#include "snac_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define NT 10  /* Tetrahedra_Count, TetrahedraTables.h:47 */

/* TetrahedraTables.c:42-84 */
static const int TetraToNode[NT][4] = {
    {7, 2, 3, 0}, {0, 5, 4, 7}, {2, 5, 1, 0}, {5, 2, 6, 7}, {2, 5, 0, 7},
    {3, 4, 7, 6}, {4, 3, 0, 1}, {6, 1, 2, 3}, {1, 6, 5, 4}, {1, 3, 6, 4}};
static const int FaceToNode[4][3] = {{0, 1, 2}, {1, 3, 2}, {0, 2, 3}, {3, 1, 0}};
static const int NodeToTetra[8][5] = {
    {3, 5, 7, 8, 9}, {0, 1, 3, 4, 5}, {1, 2, 3, 4, 8}, {1, 5, 6, 8, 9},
    {0, 2, 3, 4, 7}, {0, 5, 6, 7, 9}, {2, 6, 7, 8, 9}, {0, 1, 2, 4, 6}};
static const int NodeToSurface[8][5] = {
    {3, 0, 1, 2, 3}, {1, 0, 0, 0, 3}, {2, 2, 1, 2, 3}, {3, 2, 1, 0, 0},
    {2, 1, 2, 1, 3}, {3, 1, 2, 0, 2}, {3, 0, 2, 1, 1}, {0, 1, 0, 3, 3}};

typedef struct {
    double area;
    double normal[3];
} so_surface;

/* Snac_Element_Tetrahedra, Element.h:45-60, plus the plugin extensions of
 * that tetrahedron (plastic/Element.h, viscoplastic/Element.h,
 * maxwell/Element.h, temperature/Element.h).  The 3x3 tensors are kept whole
 * because the visco-plastic hook reads lower-triangle entries (see
 * vp_constitutive). */
typedef struct {
    double old_volume, volume;
    so_surface surface[4];
    double strainRate[3][3];
    double strain[3][3];
    double stress[3][3];
    double density, avgTemp;
    double plasticStrain, viscosity;
    double plasticstrainTensor[3][3]; /* viscoplastic/Element.h (Drucker-Prager phases) */
    double heatFlux[3], thermalStress;
} so_tet;

/* Snac_Element, Element.h:62-75 */
typedef struct {
    int material;
    double volume, strainRate, stress, hydroPressure, aps, minLengthScale;
    so_tet tet[NT];
} so_element;

struct so_ctx {
    int nx, ny, nz, nnx, nny, nnz;
    long ne, nn;
    int dt_type, constitutive, temperature, thermal_stress;
    double dt, strain_inert, gravity, demf;
    double speedOfSound, minLengthScale, initMinLengthScale, vmax;
    long timeStep;
    double currentTime; /* AbstractContext.c:871, 891 */
    int winkler;        /* SnacWinklerForce loaded */
    int traction;       /* SnacTractionBC loaded */
    double topo_kappa, topoGradCriterion, topoGradMax; /* Context.c:759-764 */
    double pisos, rzbo; /* hydroStaticIC/VariableConditions.c:120, 138 */
    double* residualFr; /* [nn] winkler/Force.c:154-161 */
    int nmat;
    snac_material* mat;
    unsigned* rheology;         /* per phase */
    int* maxiterations;         /* per phase, Context.c:851-852 */
    double* tolerance;          /* per phase, constitutivetolerance, Context.c:853-854 */
    double (*coord)[3];
    double (*vel)[3];
    double (*force)[3];
    double (*balance)[3];
    double* imass;
    double* mass;
    double* T;
    double* T0;
    so_element* el;
    unsigned char* vbc_mask;    /* bit d: component d fixed       */
    double (*vbc_val)[3];
    long* vbc_nodes;            /* velocityBCs->indexTbl           */
    long n_vbc_nodes;
    unsigned char* tbc_mask;
    double* tbc_val;
    int status;
    long err_index;
    char err[256];
};

static int fail(so_ctx* s, int code, long idx, const char* msg) {
    if (s->status == 0) {
        s->status = code;
        s->err_index = idx;
        snprintf(s->err, sizeof s->err, "%s (index %ld)", msg, idx);
    }
    return code;
}

static long nid(const so_ctx* s, int i, int j, int k) {
    return (long)i + (long)j * s->nnx + (long)k * s->nnx * s->nny;
}

/* element-local node ln of element e, HexaEL.c:456-471 */
static long enode(const so_ctx* s, long e, int ln) {
    int i = (int)(e % s->nx), j = (int)((e / s->nx) % s->ny), k = (int)(e / ((long)s->nx * s->ny));
    static const int off[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                                  {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
    return nid(s, i + off[ln][0], j + off[ln][1], k + off[ln][2]);
}

/* node -> 8 elements in HexaEL.c:529-573 order; -1 where the element is
 * outside the mesh (the reference stores elementCount and skips it, Force.c:92) */
static void node_elements(const so_ctx* s, long n, long out[8]) {
    int i = (int)(n % s->nnx), j = (int)((n / s->nnx) % s->nny), k = (int)(n / ((long)s->nnx * s->nny));
    for (int q = 0; q < 8; q++) {
        int dx = q & 1, dy = (q >> 1) & 1, dz = (q >> 2) & 1;
        int ei = i - 1 + dx, ej = j - 1 + dy, ek = k - 1 + dz;
        if (ei < 0 || ej < 0 || ek < 0 || ei >= s->nx || ej >= s->ny || ek >= s->nz)
            out[q] = -1;
        else
            out[q] = (long)ei + (long)ej * s->nx + (long)ek * s->nx * s->ny;
    }
}

/* ---- Tetrahedra.c:44-113 -------------------------------------------------- */
double so_tetrahedra_volume(const double* c1, const double* c2, const double* c3, const double* c4) {
    double x2 = c2[0] - c1[0], y2 = c2[1] - c1[1], z2 = c2[2] - c1[2];
    double x3 = c3[0] - c1[0], y3 = c3[1] - c1[1], z3 = c3[2] - c1[2];
    double x4 = c4[0] - c1[0], y4 = c4[1] - c1[1], z4 = c4[2] - c1[2];
    double volume = (x4 * (y2 * z3 - z2 * y3) + y4 * (z2 * x3 - x2 * z3) + z4 * (x2 * y3 - x3 * y2)) / 6.0;
    return fabs(volume);
}

double so_tetrahedra_surface_area(const double* c1, const double* c2, const double* c3) {
    double x2 = c2[0] - c1[0], y2 = c2[1] - c1[1], z2 = c2[2] - c1[2];
    double x3 = c3[0] - c1[0], y3 = c3[1] - c1[1], z3 = c3[2] - c1[2];
    double a = y2 * z3 - z2 * y3;
    double b = z2 * x3 - x2 * z3;
    double c = x2 * y3 - y2 * x3;
    return sqrt(a * a + b * b + c * c) / 2.0f;
}

void so_tetrahedra_surface_normal(const double* c1, const double* c2, const double* c3, double* n) {
    double x2 = c2[0] - c1[0], y2 = c2[1] - c1[1], z2 = c2[2] - c1[2];
    double x3 = c3[0] - c1[0], y3 = c3[1] - c1[1], z3 = c3[2] - c1[2];
    double ax = y2 * z3 - z2 * y3;
    double ay = z2 * x3 - x2 * z3;
    double az = x2 * y3 - y2 * x3;
    double aa = 1. * sqrt(ax * ax + ay * ay + az * az);
    n[0] = +1.0f * ax / aa;
    n[1] = +1.0f * ay / aa;
    n[2] = +1.0f * az / aa;
}

/* ---- principal stresses: plastic/Constitutive.c:249-410 (Numerical
 * Recipes cyclic Jacobi, eigsrt), restated with 0-based indices ----------- */
#define SO_ROTATE(a, i, j, k, l)                 \
    do {                                         \
        g = a[i][j];                             \
        h = a[k][l];                             \
        a[i][j] = g - s * (h + g * tau);         \
        a[k][l] = h + s * (g - h * tau);         \
    } while (0)

static void so_jacobi(double a[3][3], double d[3], double v[3][3]) {
    const unsigned n = 3;
    double b[3], z[3], tresh, sm, g, h, t, theta, c, s, tau;
    int i, j, ip, iq;
    for (ip = 0; ip < 3; ip++) {
        for (iq = 0; iq < 3; iq++) v[ip][iq] = 0.0f;
        v[ip][ip] = 1.0f;
    }
    for (ip = 0; ip < 3; ip++) {
        b[ip] = d[ip] = a[ip][ip];
        z[ip] = 0.0f;
    }
    for (i = 1; i <= 50; i++) {
        sm = 0.0f;
        for (ip = 0; ip < 2; ip++)
            for (iq = ip + 1; iq < 3; iq++) sm += fabs(a[ip][iq]);
        if (sm == 0.0f) return;
        if (i < 4)
            tresh = 0.2f * sm / (n * n);
        else
            tresh = 0.0f;
        for (ip = 0; ip < 2; ip++) {
            for (iq = ip + 1; iq < 3; iq++) {
                g = 100.0f * fabs(a[ip][iq]);
                if ((i > 4) && (double)(fabs(d[ip]) + g) == (double)fabs(d[ip]) &&
                    (double)(fabs(d[iq]) + g) == (double)fabs(d[iq]))
                    a[ip][iq] = 0.0f;
                else if (fabs(a[ip][iq]) > tresh) {
                    h = d[iq] - d[ip];
                    if ((fabs(h) + g) == fabs(h))
                        t = a[ip][iq] / h;
                    else {
                        theta = 0.5f * h / (a[ip][iq]);
                        t = 1.0f / (fabs(theta) + sqrt(1.0f + theta * theta));
                        if (theta < 0.0f) t *= -1.0f;
                    }
                    c = 1.0f / sqrt(1.0f + t * t);
                    s = t * c;
                    tau = s / (1.0f + c);
                    h = t * a[ip][iq];
                    z[ip] -= h;
                    z[iq] += h;
                    d[ip] -= h;
                    d[iq] += h;
                    a[ip][iq] = 0.0f;
                    for (j = 0; j <= ip - 1; j++) SO_ROTATE(a, j, ip, j, iq);
                    for (j = ip + 1; j <= iq - 1; j++) SO_ROTATE(a, ip, j, j, iq);
                    for (j = iq + 1; j < 3; j++) SO_ROTATE(a, ip, j, iq, j);
                    for (j = 0; j < 3; j++) SO_ROTATE(v, j, ip, j, iq);
                }
            }
        }
        for (ip = 0; ip < 3; ip++) {
            b[ip] += z[ip];
            d[ip] = b[ip];
            z[ip] = 0.0f;
        }
    }
}

static void so_eigsrt(double d[3], double v[3][3]) {
    for (int i = 0; i < 2; i++) {
        int k = i;
        double p = d[i];
        for (int j = i + 1; j < 3; j++)
            if (d[j] >= p) {
                k = j;
                p = d[j];
            }
        if (k != i) {
            d[k] = d[i];
            d[i] = p;
            for (int j = 0; j < 3; j++) {
                p = v[j][i];
                v[j][i] = v[j][k];
                v[j][k] = p;
            }
        }
    }
}

static void principal(double st[3][3], double sp[3], double cn[3][3]) {
    double a[3][3], v[3][3], d[3];
    a[0][0] = st[0][0];
    a[1][1] = st[1][1];
    a[2][2] = st[2][2];
    a[0][1] = st[0][1];
    a[0][2] = st[0][2];
    a[1][2] = st[1][2];
    a[1][0] = a[0][1];
    a[2][0] = a[0][2];
    a[2][1] = a[1][2];
    so_jacobi(a, d, v);
    d[0] *= -1.0f;
    d[1] *= -1.0f;
    d[2] *= -1.0f;
    so_eigsrt(d, v);
    d[0] *= -1.0f;
    d[1] *= -1.0f;
    d[2] *= -1.0f;
    for (int i = 0; i < 3; i++) {
        sp[i] = d[i];
        for (int j = 0; j < 3; j++) cn[i][j] = v[j][i];
    }
}

void so_principal_stresses(const double* s6, double* s, double* cn) {
    double st[3][3] = {{s6[0], s6[3], s6[4]}, {0, s6[1], s6[5]}, {0, 0, s6[2]}};
    double c[3][3];
    principal(st, s, c);
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) cn[i * 3 + j] = c[i][j];
}

/* ---- material helpers ---------------------------------------------------- */
static double degrad_of(void) { return 3.14159265358979323846 / 180.0f; }

/* ---- UpdateElement.c:54-269 ----------------------------------------------- */
static void update_element(so_ctx* s, long e, double* minLS) {
    so_element* el = &s->el[e];
    const snac_material* m = &s->mat[el->material];
    double rotation[NT][3][3];
    if (s->dt_type == SNAC_DT_WAVE) {
        double Vp = sqrt((m->lambda + 2.0f * m->mu) / m->density);
        if (Vp > s->speedOfSound) s->speedOfSound = Vp;
    }
    el->volume = 0.0;
    *minLS = 1.0e+27f;
    memset(rotation, 0, sizeof rotation);
    for (int t = 0; t < NT; t++) {
        so_tet* tt = &el->tet[t];
        const double* c[4];
        const double* v[4];
        for (int q = 0; q < 4; q++) {
            long n = enode(s, e, TetraToNode[t][q]);
            c[q] = s->coord[n];
            v[q] = s->vel[n];
        }
        memset(tt->strain, 0, sizeof tt->strain);
        tt->old_volume = tt->volume;
        tt->volume = so_tetrahedra_volume(c[0], c[1], c[2], c[3]);
        if (s->timeStep == 0) tt->old_volume = tt->volume;
        for (int f = 0; f < 4; f++) {
            tt->surface[f].area = so_tetrahedra_surface_area(c[FaceToNode[f][0]], c[FaceToNode[f][1]], c[FaceToNode[f][2]]);
            so_tetrahedra_surface_normal(c[FaceToNode[f][0]], c[FaceToNode[f][1]], c[FaceToNode[f][2]],
                                         tt->surface[f].normal);
        }
        for (int f = 0; f < 4; f++) {
            double ls = tt->surface[f].area;
            if (ls) {
                ls = fabs(tt->volume / ls);
                if (*minLS > ls) *minLS = ls;
            }
        }
        el->volume += tt->volume;
        {
            const so_surface* S = tt->surface;
            double V = tt->volume;
            double (*r)[3] = rotation[t];
            r[0][1] = -(0.5f / V) *
                      (v[0][0] * S[1].normal[1] * S[1].area + v[1][0] * S[2].normal[1] * S[2].area +
                       v[2][0] * S[3].normal[1] * S[3].area + v[3][0] * S[0].normal[1] * S[0].area -
                       v[0][1] * S[1].normal[0] * S[1].area - v[1][1] * S[2].normal[0] * S[2].area -
                       v[2][1] * S[3].normal[0] * S[3].area - v[3][1] * S[0].normal[0] * S[0].area) /
                      3.0f;
            r[0][2] = -(0.5f / V) *
                      (v[0][0] * S[1].normal[2] * S[1].area + v[1][0] * S[2].normal[2] * S[2].area +
                       v[2][0] * S[3].normal[2] * S[3].area + v[3][0] * S[0].normal[2] * S[0].area -
                       v[0][2] * S[1].normal[0] * S[1].area - v[1][2] * S[2].normal[0] * S[2].area -
                       v[2][2] * S[3].normal[0] * S[3].area - v[3][2] * S[0].normal[0] * S[0].area) /
                      3.0f;
            r[1][2] = -(0.5 / V) *
                      (v[0][1] * S[1].normal[2] * S[1].area + v[1][1] * S[2].normal[2] * S[2].area +
                       v[2][1] * S[3].normal[2] * S[3].area + v[3][1] * S[0].normal[2] * S[0].area -
                       v[0][2] * S[1].normal[1] * S[1].area - v[1][2] * S[2].normal[1] * S[2].area -
                       v[2][2] * S[3].normal[1] * S[3].area - v[3][2] * S[0].normal[1] * S[0].area) /
                      3.0f;
            double dt = s->dt;
            double (*e3)[3] = tt->strain;
            /* strain rotation (UpdateElement.c:222-240; strain was just zeroed) */
            e3[0][0] += (2.0f * r[0][1] * e3[0][1] + 2.0f * r[0][2] * e3[0][2]) * dt;
            e3[1][1] += (2.0f * (-1.0f * r[0][1]) * e3[0][1] + 2.0f * r[1][2] * e3[1][2]) * dt;
            e3[2][2] += (2.0f * (-1.0f * r[0][2]) * e3[0][2] + 2.0f * (-1.0f * r[1][2]) * e3[1][2]) * dt;
            e3[0][1] += (r[0][1] * (e3[1][1] - e3[0][0])) * dt + (r[0][2] * e3[1][2] - r[1][2] * e3[0][2]) * dt;
            e3[0][2] += (r[0][2] * (e3[2][2] - e3[0][0])) * dt + (r[0][1] * e3[1][2] - r[0][2] * e3[0][1]) * dt;
            e3[1][2] += (r[1][2] * (e3[2][2] - e3[1][1])) * dt + ((-1.0f * r[0][1]) * e3[0][2] - r[0][2] * e3[0][1]) * dt;
            /* stress rotation (UpdateElement.c:243-265): note "+ r12*s02" in s01 */
            double (*s3)[3] = tt->stress;
            s3[0][0] += (2.0f * r[0][1] * s3[0][1] + 2.0f * r[0][2] * s3[0][2]) * dt;
            s3[1][1] += (2.0f * (-1.0f * r[0][1]) * s3[0][1] + 2.0f * r[1][2] * s3[1][2]) * dt;
            s3[2][2] += (2.0f * (-1.0f * r[0][2]) * s3[0][2] + 2.0f * (-1.0f * r[1][2]) * s3[1][2]) * dt;
            s3[0][1] += (r[0][1] * (s3[1][1] - s3[0][0])) * dt + (r[0][2] * s3[1][2] + r[1][2] * s3[0][2]) * dt;
            s3[0][2] += (r[0][2] * (s3[2][2] - s3[0][0])) * dt + (r[0][1] * s3[1][2] - r[1][2] * s3[0][1]) * dt;
            s3[1][2] += (r[1][2] * (s3[2][2] - s3[1][1])) * dt + ((-1.0f * r[0][1]) * s3[0][2] - r[0][2] * s3[0][1]) * dt;
        }
    }
    el->volume *= 0.5;
    el->minLengthScale = *minLS;
}

/* ---- StrainRate.c:49-305 ---------------------------------------------------- */
static void strain_rate(so_ctx* s, long e) {
    so_element* el = &s->el[e];
    double trace[NT], partial, volAvg, otherAvg;
    double elemVolume = 2.0 * el->volume;
    for (int t = 0; t < NT; t++) {
        so_tet* tt = &el->tet[t];
        const double* v[4];
        for (int q = 0; q < 4; q++) v[q] = s->vel[enode(s, e, TetraToNode[t][q])];
        const so_surface* S = tt->surface;
        double (*sr)[3] = tt->strainRate;
        memset(sr, 0, sizeof tt->strainRate);
        for (int d = 0; d < 3; d++)
            sr[d][d] = -1.0f *
                       (v[0][d] * S[1].normal[d] * S[1].area + v[1][d] * S[2].normal[d] * S[2].area +
                        v[2][d] * S[3].normal[d] * S[3].area + v[3][d] * S[0].normal[d] * S[0].area) /
                       3.0f / tt->volume;
        static const int pr[3][2] = {{0, 1}, {0, 2}, {1, 2}};
        for (int p = 0; p < 3; p++) {
            int a = pr[p][0], b = pr[p][1];
            sr[a][b] = -0.5f *
                       (v[0][a] * S[1].normal[b] * S[1].area + v[1][a] * S[2].normal[b] * S[2].area +
                        v[2][a] * S[3].normal[b] * S[3].area + v[3][a] * S[0].normal[b] * S[0].area +
                        v[0][b] * S[1].normal[a] * S[1].area + v[1][b] * S[2].normal[a] * S[2].area +
                        v[2][b] * S[3].normal[a] * S[3].area + v[3][b] * S[0].normal[a] * S[0].area) /
                       3.0f / tt->volume;
        }
    }
    partial = 0.0f;
    for (int t = 0; t < NT; t++) {
        so_tet* tt = &el->tet[t];
        trace[t] = (tt->strainRate[0][0] + tt->strainRate[1][1] + tt->strainRate[2][2]) / 3.0f;
        partial += trace[t] * tt->volume;
    }
    volAvg = 0.0f;
    otherAvg = 0.0f;
    for (int t = 0; t < NT; t++) {
        double (*sr)[3] = el->tet[t].strainRate;
        sr[0][0] += -1.0f * trace[t] + partial / elemVolume;
        sr[1][1] += -1.0f * trace[t] + partial / elemVolume;
        sr[2][2] += -1.0f * trace[t] + partial / elemVolume;
        volAvg += sr[1][1] * sr[2][2] + sr[2][2] * sr[0][0] + sr[0][0] * sr[1][1];
        otherAvg += sr[0][1] * sr[0][1] + sr[1][2] * sr[1][2] + sr[0][2] * sr[0][2];
    }
    volAvg /= NT;
    otherAvg /= NT;
    el->strainRate = 0.5f * sqrt(0.5f * fabs(-1.0f * volAvg + otherAvg));
    for (int t = 0; t < NT; t++)
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++)
                if (!isfinite(el->tet[t].strainRate[a][b])) fail(s, SNAC_GPU_ENAN, e, "strain rate is nan or inf");
}

/* ---- elastic/Constitutive.c:40-66 ------------------------------------------ */
static void elastic_constitutive(so_ctx* s, long e) {
    so_element* el = &s->el[e];
    const snac_material* m = &s->mat[el->material];
    if (!(s->rheology[el->material] & SNAC_RHEOLOGY_ELASTIC)) return;
    for (int t = 0; t < NT; t++) {
        const double a2 = m->lambda;
        const double sh2 = 2.0 * m->mu;
        double (*st)[3] = el->tet[t].stress;
        double (*sn)[3] = el->tet[t].strain;
        double trace_strain = sn[0][0] + sn[1][1] + sn[2][2];
        st[0][0] += sh2 * sn[0][0] + a2 * (trace_strain);
        st[1][1] += sh2 * sn[1][1] + a2 * (trace_strain);
        st[2][2] += sh2 * sn[2][2] + a2 * (trace_strain);
        st[0][1] += sh2 * sn[0][1];
        st[0][2] += sh2 * sn[0][2];
        st[1][2] += sh2 * sn[1][2];
    }
}

/* Mohr-Coulomb return map shared by plastic/Constitutive.c:180-237 and
 * viscoplastic/Constitutive.c:305-370 (identical arithmetic in both). */
static int mc_return_map(double sp[3], double cn[3][3], double (*stress)[3], double* plasticStrain,
                         double cohesion, double hardening, double anphi, double anpsi, double st,
                         double a1, double a2) {
    double alam, dep1, dep2, dep3, depm, fs, ft, aP, sP, h;
    int ind = 0;
    fs = sp[0] - sp[2] * anphi + 2 * cohesion * sqrt(anphi);
    ft = sp[2] - st;
    if (fs < 0.0f || ft > 0.0f) {
        ind = 1;
        aP = sqrt(1.0f + anphi * anphi) + anphi;
        sP = st * anphi - 2 * cohesion * sqrt(anphi);
        h = sp[2] - st + aP * (sp[0] - sP);
        if (h < 0.0f) {
            alam = fs / (a1 - a2 * anpsi + a1 * anphi * anpsi - a2 * anphi + 2.0 * sqrt(anphi) * hardening);
            sp[0] -= alam * (a1 - a2 * anpsi);
            sp[1] -= alam * a2 * (1.0f - anpsi);
            sp[2] -= alam * (a2 - a1 * anpsi);
            dep1 = alam;
            dep2 = 0.0f;
            dep3 = -alam * anpsi;
        } else {
            alam = ft / a1;
            sp[0] -= alam * a2;
            sp[1] -= alam * a2;
            sp[2] -= alam * a1;
            dep1 = 0.0f;
            dep2 = 0.0f;
            dep3 = alam;
        }
    } else {
        dep1 = 0.0f;
        dep2 = 0.0f;
        dep3 = 0.0f;
    }
    if (ind) {
        depm = (dep1 + dep2 + dep3) / 3.0f;
        *plasticStrain += sqrt(0.5f * ((dep1 - depm) * (dep1 - depm) + (dep2 - depm) * (dep2 - depm) +
                                       (dep3 - depm) * (dep3 - depm) + depm * depm));
        memset(stress, 0, sizeof(double[3][3]));
        for (int mm = 0; mm < 3; mm++)
            for (int nn = mm; nn < 3; nn++)
                for (int k = 0; k < 3; k++) stress[mm][nn] += cn[k][mm] * cn[k][nn] * sp[k];
    }
    return ind;
}

/* ---- plastic/Constitutive.c:58-247 ----------------------------------------- */
static void plastic_constitutive(so_ctx* s, long e) {
    so_element* el = &s->el[e];
    const snac_material* m = &s->mat[el->material];
    if (!(s->rheology[el->material] & SNAC_RHEOLOGY_PLASTIC)) return;
    double cohesion = 0.0f, frictionAngle = 0.0f, dilationAngle = 0.0f, hardening = 0.0f;
    double sphi = 0.0f, spsi = 0.0f, st = 0.0f;
    const double degrad = degrad_of();
    double totalVolume = 0.0f, depls = 0.0f, tmp = 0.0f, anphi = 0.0f, anpsi = 0.0f;
    const double a1 = m->lambda + 2.0f * m->mu;
    const double a2 = m->lambda;
    for (int t = 0; t < NT; t++) {
        so_tet* tt = &el->tet[t];
        double cn[3][3] = {{0}}, sp[3] = {0};
        double (*stress)[3] = tt->stress;
        double (*strain)[3] = tt->strain;
        double plasticStrain = tt->plasticStrain;
        double trace_strain = strain[0][0] + strain[1][1] + strain[2][2];
        stress[0][0] += (2.0f * m->mu) * strain[0][0] + m->lambda * (trace_strain);
        stress[1][1] += (2.0f * m->mu) * strain[1][1] + m->lambda * (trace_strain);
        stress[2][2] += (2.0f * m->mu) * strain[2][2] + m->lambda * (trace_strain);
        stress[0][1] += (2.0f * m->mu) * strain[0][1];
        stress[0][2] += (2.0f * m->mu) * strain[0][2];
        stress[1][2] += (2.0f * m->mu) * strain[1][2];
        principal(stress, sp, cn);
        if (m->plstrain[0] != 0.0) fail(s, SNAC_GPU_EINVAL, e, "initial softening segment must start at 0");
        for (int i = 0; i < m->nsegments; i++) {
            const double pl1 = m->plstrain[i];
            const double pl2 = m->plstrain[i + 1];
            if (plasticStrain >= pl1 && plasticStrain <= pl2) {
                const double tgf = (m->friction_angle[i + 1] - m->friction_angle[i]) / (pl2 - pl1);
                const double tgd = (m->dilation_angle[i + 1] - m->dilation_angle[i]) / (pl2 - pl1);
                const double tgc = (m->cohesion[i + 1] - m->cohesion[i]) / (pl2 - pl1);
                frictionAngle = m->friction_angle[i] + tgf * (plasticStrain - pl1);
                dilationAngle = m->dilation_angle[i] + tgd * (plasticStrain - pl1);
                cohesion = m->cohesion[i] + tgc * (plasticStrain - pl1);
                hardening = tgc;
                break;
            } else if (i == m->nsegments - 1 && plasticStrain > pl2) {
                frictionAngle = m->friction_angle[m->nsegments];
                dilationAngle = m->dilation_angle[m->nsegments];
                cohesion = m->cohesion[m->nsegments];
                hardening = 0.0;
                break;
            }
        }
        sphi = sin(frictionAngle * degrad);
        spsi = sin(dilationAngle * degrad);
        anphi = (1.0f + sphi) / (1.0f - sphi);
        anpsi = (1.0f + spsi) / (1.0f - spsi);
        if (frictionAngle >= 0.0f) {
            st = m->ten_off;
            if (frictionAngle > 0.0) {
                tmp = cohesion / tan(frictionAngle * degrad);
                if (tmp < st) st = tmp;
            }
        } else {
            fail(s, SNAC_GPU_EPHYSICS, e, "friction angle < 0 (plastic abort)");
            return;
        }
        mc_return_map(sp, cn, stress, &tt->plasticStrain, cohesion, hardening, anphi, anpsi, st, a1, a2);
        depls += tt->plasticStrain * tt->volume;
        totalVolume += tt->volume;
    }
    el->aps = depls / totalVolume;
}

/* ---- viscoplastic/Constitutive.c:61-525 (Mohr-Coulomb branch) -------------- */
/* viscoplastic/Constitutive.c:372-518: the Drucker-Prager return map of one
 * tetrahedron, after its viscous update.  sd holds the updated deviatoric
 * diagonal, Stress0 the stress before the viscous update.  Up to
 * maxiterations passes: from the shear (h > 0) or tension branch, the
 * plastic strain increments; with more than one pass the viscous update is
 * redone with them and the yield functions re-evaluated until both fall
 * below tolerance times their larger first value.  The increments accumulate
 * in the plastic strain tensor, whose second invariant becomes the plastic
 * strain.  palam (the previous pass's multiplier, used when a pass gives a
 * negative one) is an uninitialised variable of the reference's function on
 * its first use; it starts at 0 here. */
static void dp_return_map(double (*stress)[3], double sd[3], double Stress0[3][3], double (*strain)[3], double vic1,
                          double vic2, double rmu, double bulkm, double qphi, double qpsi, double kphi, double st,
                          double tolerance, int mite, double (*pst)[3], double* plasticStrain) {
    double I1 = (stress[0][0] + stress[1][1] + stress[2][2]) / 3.;
    double J2 = sqrt(0.5 * (sd[0] * sd[0] + sd[1] * sd[1] + sd[2] * sd[2]) + stress[0][1] * stress[0][1] +
                     stress[0][2] * stress[0][2] + stress[1][2] * stress[1][2]);
    double fs = J2 + I1 * qphi - kphi;
    double ft = I1 - st;
    if (!(fs > 0.0f || ft > 0.0f)) return;
    double dep0 = 0.0, dep1 = 0.0, dep2 = 0.0, dep01 = 0.0, dep02 = 0.0, dep12 = 0.0, depm;
    const double tolerf = fs > ft ? tolerance * fs : tolerance * ft;
    double previousfs = fs, previousft = ft, palam = 0.0, alam;
    for (int ite = 0; ite < mite; ite++) {
        const double aP = sqrt(1.0f + qphi * qphi) - qphi;
        const double sP = kphi - qphi * st;
        const double h = J2 - sP - aP * (I1 - st);
        if (h > 0.0f) {
            alam = fs / (bulkm * qphi * qpsi + rmu);
            if (alam < 0.0) alam = palam * (previousfs / (previousfs - fs));
            dep0 = alam * (0.5 * sd[0] / J2 + qpsi / 3.);
            dep1 = alam * (0.5 * sd[1] / J2 + qpsi / 3.);
            dep2 = alam * (0.5 * sd[2] / J2 + qpsi / 3.);
            dep01 = alam * 0.5 * (stress[0][1]) / J2;
            dep02 = alam * 0.5 * (stress[0][2]) / J2;
            dep12 = alam * 0.5 * (stress[1][2]) / J2;
        } else {
            alam = ft / bulkm;
            if (alam < 0.0) alam = palam * (previousft / (previousfs - ft));
            dep0 = alam / 3.;
            dep1 = alam / 3.;
            dep2 = alam / 3.;
        }
        if (mite == 1) break;
        depm = (dep0 + dep1 + dep2) / 3.0f;
        const double trace_strain = strain[0][0] + strain[1][1] + strain[2][2];
        const double straind0 = strain[0][0] - dep0 - (trace_strain) / 3.0f + depm;
        const double straind1 = strain[1][1] - dep1 - (trace_strain) / 3.0f + depm;
        const double straind2 = strain[2][2] - dep2 - (trace_strain) / 3.0f + depm;
        const double trace_stress = Stress0[0][0] + Stress0[1][1] + Stress0[2][2];
        sd[0] = Stress0[0][0] - trace_stress / 3.;
        sd[1] = Stress0[1][1] - trace_stress / 3.;
        sd[2] = Stress0[2][2] - trace_stress / 3.;
        sd[0] = (sd[0] * vic1 + 2.0f * rmu * straind0) * vic2;
        sd[1] = (sd[1] * vic1 + 2.0f * rmu * straind1) * vic2;
        sd[2] = (sd[2] * vic1 + 2.0f * rmu * straind2) * vic2;
        stress[0][1] = (Stress0[0][1] * vic1 + 2.0f * rmu * (strain[0][1] - dep01)) * vic2;
        stress[0][2] = (Stress0[0][2] * vic1 + 2.0f * rmu * (strain[0][2] - dep02)) * vic2;
        stress[1][2] = (Stress0[1][2] * vic1 + 2.0f * rmu * (strain[1][2] - dep12)) * vic2;
        const double VolumicStress = trace_stress / 3.0f + bulkm * (trace_strain - 3. * depm);
        stress[0][0] = sd[0] + VolumicStress;
        stress[1][1] = sd[1] + VolumicStress;
        stress[2][2] = sd[2] + VolumicStress;
        I1 = (stress[0][0] + stress[1][1] + stress[2][2]) / 3.;
        sd[0] = stress[0][0] - I1;
        sd[1] = stress[1][1] - I1;
        sd[2] = stress[2][2] - I1;
        J2 = sqrt(0.5 * (sd[0] * sd[0] + sd[1] * sd[1] + sd[2] * sd[2]) + stress[0][1] * stress[0][1] +
                  stress[0][2] * stress[0][2] + stress[1][2] * stress[1][2]);
        previousfs = fs;
        previousft = ft;
        palam = alam;
        fs = J2 + I1 * qphi - kphi;
        ft = I1 - st;
        if (fs < tolerf && ft < tolerf) break;
    }
    pst[0][0] += dep0;
    pst[1][1] += dep1;
    pst[2][2] += dep2;
    pst[0][1] += dep01;
    pst[0][2] += dep02;
    pst[1][2] += dep12;
    depm = (pst[0][0] + pst[1][1] + pst[2][2]) / 3.0f;
    *plasticStrain = sqrt(0.5f * ((pst[0][0] - depm) * (pst[0][0] - depm) + (pst[1][1] - depm) * (pst[1][1] - depm) +
                                  (pst[2][2] - depm) * (pst[2][2] - depm)) +
                          pst[0][1] * pst[0][1] + pst[0][2] * pst[0][2] + pst[1][2] * pst[1][2]);
}

static void vp_constitutive(so_ctx* s, long e) {
    so_element* el = &s->el[e];
    const snac_material* m = &s->mat[el->material];
    if (!(s->rheology[el->material] & SNAC_RHEOLOGY_VISCOPLASTIC)) return;
    const double bulkm = m->lambda + 2.0f * m->mu / 3.0f;
    double straind0, straind1, straind2, stressd0, stressd1, stressd2;
    double trace_strain, trace_stress, temp, vic1, vic2, VolumicStress;
    double rviscosity = m->refvisc, rmu = m->mu, srJ2, avgTemp;
    double rstrainrate = m->refsrate, rTemp = m->reftemp, H = m->activation_e, srexponent = m->srexponent;
    const double R = 8.31448;
    double cohesion = 0.0f, frictionAngle = 0.0f, dilationAngle = 0.0f, hardening = 0.0f;
    double sphi = 0.0, spsi = 0.0, st = 0.0;
    const double degrad = degrad_of();
    double totalVolume = 0.0f, depls = 0.0f, tmp = 0.0, anphi = 0.0, anpsi = 0.0;
    const double a1 = m->lambda + 2.0f * m->mu;
    const double a2 = m->lambda;
    for (int t = 0; t < NT; t++) {
        so_tet* tt = &el->tet[t];
        double cn[3][3] = {{0}}, sp[3] = {0};
        double (*stress)[3] = tt->stress;
        double (*strain)[3] = tt->strain;
        double plasticStrain = tt->plasticStrain;
        if (s->thermal_stress) {
            stress[0][0] += tt->thermalStress;
            stress[1][1] += tt->thermalStress;
            stress[2][2] += tt->thermalStress;
        }
        /* the stress before the viscous update (Stress0, :165-170) */
        double Stress0[3][3];
        memcpy(Stress0, stress, sizeof Stress0);
        trace_stress = stress[0][0] + stress[1][1] + stress[2][2];
        trace_strain = strain[0][0] + strain[1][1] + strain[2][2];
        straind0 = strain[0][0] - (trace_strain) / 3.0f;
        straind1 = strain[1][1] - (trace_strain) / 3.0f;
        straind2 = strain[2][2] - (trace_strain) / 3.0f;
        stressd0 = stress[0][0] - (trace_stress) / 3.0f;
        stressd1 = stress[1][1] - (trace_stress) / 3.0f;
        stressd2 = stress[2][2] - (trace_stress) / 3.0f;
        /* viscoplastic/Constitutive.c:189: "(*strain[0][1])" and friends index
         * the pointer, not the tensor: they read strain[1][0], strain[2][0] and
         * (one tensor past strain, i.e. the stress) stress[2][0].  Those
         * lower-triangle entries are never written, so the shear terms of the
         * second invariant vanish. */
        srJ2 = sqrt(fabs(straind1 * straind2 + straind2 * straind0 + straind0 * straind1 -
                         (strain[1][0]) * (strain[1][0]) - (strain[2][0]) * (strain[2][0]) -
                         (stress[2][0]) * (stress[2][0]))) /
               s->dt;
        if (srJ2 == 0.0f) srJ2 = rstrainrate;
        avgTemp = 0.0;
        for (int q = 0; q < 4; q++) avgTemp += 0.25 * s->T[enode(s, e, TetraToNode[t][q])];
        tt->viscosity = rviscosity * pow((srJ2 / rstrainrate), (1. / srexponent - 1.)) *
                        exp(H / R * (1. / (avgTemp + 273.15) - 1. / (rTemp + 273.15)));
        if (tt->viscosity < m->vis_min) tt->viscosity = m->vis_min;
        if (tt->viscosity > m->vis_max) tt->viscosity = m->vis_max;
        if (!isfinite(tt->viscosity)) fail(s, SNAC_GPU_ENAN, e, "viscosity is nan or inf");
        temp = rmu / (2.0f * (tt->viscosity)) * s->dt;
        vic1 = 1.0f - temp;
        vic2 = 1.0f / (1.0f + temp);
        stressd0 = (stressd0 * vic1 + 2.0f * rmu * straind0) * vic2;
        stressd1 = (stressd1 * vic1 + 2.0f * rmu * straind1) * vic2;
        stressd2 = (stressd2 * vic1 + 2.0f * rmu * straind2) * vic2;
        stress[0][1] = (stress[0][1] * vic1 + 2.0f * rmu * strain[0][1]) * vic2;
        stress[0][2] = (stress[0][2] * vic1 + 2.0f * rmu * strain[0][2]) * vic2;
        stress[1][2] = (stress[1][2] * vic1 + 2.0f * rmu * strain[1][2]) * vic2;
        VolumicStress = trace_stress / 3.0f + bulkm * trace_strain;
        stress[0][0] = stressd0 + VolumicStress;
        stress[1][1] = stressd1 + VolumicStress;
        stress[2][2] = stressd2 + VolumicStress;
        principal(stress, sp, cn);
        /* softening table without break or clamp (:279-293); the values carry
         * over from the previous tetrahedron when no segment matches */
        for (int i = 0; i < m->nsegments; i++) {
            const double pl1 = m->plstrain[i];
            const double pl2 = m->plstrain[i + 1];
            if (plasticStrain >= pl1 && plasticStrain <= pl2) {
                const double tgf = (m->friction_angle[i + 1] - m->friction_angle[i]) / (pl2 - pl1);
                const double tgd = (m->dilation_angle[i + 1] - m->dilation_angle[i]) / (pl2 - pl1);
                const double tgc = (m->cohesion[i + 1] - m->cohesion[i]) / (pl2 - pl1);
                frictionAngle = m->friction_angle[i] + tgf * (plasticStrain - pl1);
                dilationAngle = m->dilation_angle[i] + tgd * (plasticStrain - pl1);
                cohesion = m->cohesion[i] + tgc * (plasticStrain - pl1);
                hardening = tgc;
            }
        }
        if (frictionAngle > 0.0f) {
            st = m->ten_off;
            if (frictionAngle > 0.0) {
                tmp = cohesion / tan(frictionAngle * degrad);
                if (tmp < st) st = tmp;
            }
        } /* else: assert(0), compiled out of the -DNDEBUG reference build */
        if (m->yield_mohr_coulomb) {
            sphi = sin(frictionAngle * degrad);
            spsi = sin(dilationAngle * degrad);
            anphi = (1.0f + sphi) / (1.0f - sphi);
            anpsi = (1.0f + spsi) / (1.0f - spsi);
            mc_return_map(sp, cn, stress, &tt->plasticStrain, cohesion, hardening, anphi, anpsi, st, a1, a2);
        } else {
            double sd[3] = {stressd0, stressd1, stressd2};
            dp_return_map(stress, sd, Stress0, strain, vic1, vic2, rmu, bulkm, tan(frictionAngle * degrad),
                          tan(dilationAngle * degrad), cohesion, st, s->tolerance[el->material],
                          s->maxiterations[el->material], tt->plasticstrainTensor, &tt->plasticStrain);
        }
        depls += tt->plasticStrain * tt->volume;
        totalVolume += tt->volume;
    }
    el->aps = depls / totalVolume;
}

/* ---- maxwell/Constitutive.c:47-184 ------------------------------------------ */
static void maxwell_constitutive(so_ctx* s, long e) {
    so_element* el = &s->el[e];
    const snac_material* m = &s->mat[el->material];
    if (!(s->rheology[el->material] & SNAC_RHEOLOGY_MAXWELL)) return;
    for (int t = 0; t < NT; t++) {
        so_tet* tt = &el->tet[t];
        const double bulkm = m->lambda + 2.0f * m->mu / 3.0f;
        double (*stress)[3] = tt->stress;
        double (*strain)[3] = tt->strain;
        double straind0, straind1, straind2, stressd0, stressd1, stressd2;
        double trace_strain, trace_stress, temp, vic1, vic2, VolumicStress;
        double rviscosity = m->refvisc, rmu = m->mu, srJ2, avgTemp;
        double rstrainrate = m->refsrate, rTemp = m->reftemp, H = m->activation_e, srexponent = m->srexponent;
        const double R = 8.31448;
        if (s->thermal_stress) {
            stress[0][0] += tt->thermalStress;
            stress[1][1] += tt->thermalStress;
            stress[2][2] += tt->thermalStress;
        }
        trace_stress = stress[0][0] + stress[1][1] + stress[2][2];
        trace_strain = tt->volume / tt->old_volume - 1.0f;
        straind0 = strain[0][0] - (trace_strain) / 3.0f;
        straind1 = strain[1][1] - (trace_strain) / 3.0f;
        straind2 = strain[2][2] - (trace_strain) / 3.0f;
        stressd0 = stress[0][0] - (trace_stress) / 3.0f;
        stressd1 = stress[1][1] - (trace_stress) / 3.0f;
        stressd2 = stress[2][2] - (trace_stress) / 3.0f;
        srJ2 = sqrt(fabs(straind1 * straind2 + straind2 * straind0 + straind0 * straind1 -
                         strain[0][1] * strain[0][1] - strain[0][2] * strain[0][2] - strain[1][2] * strain[1][2])) /
               s->dt;
        if (srJ2 == 0.0f) srJ2 = rstrainrate;
        avgTemp = 0.0;
        for (int q = 0; q < 4; q++) avgTemp += 0.25 * s->T[enode(s, e, TetraToNode[t][q])];
        tt->viscosity = rviscosity * pow((srJ2 / rstrainrate), (1. / srexponent - 1.)) *
                        exp(H / R * (1. / (avgTemp + 273.15) - 1. / (rTemp + 273.15)));
        if (tt->viscosity < m->vis_min) tt->viscosity = m->vis_min;
        if (tt->viscosity > m->vis_max) tt->viscosity = m->vis_max;
        if (!isfinite(tt->viscosity)) fail(s, SNAC_GPU_ENAN, e, "viscosity is nan or inf");
        temp = rmu / (2.0f * (tt->viscosity)) * s->dt;
        vic1 = 1.0f - temp;
        vic2 = 1.0f / (1.0f + temp);
        stressd0 = (stressd0 * vic1 + 2.0f * rmu * straind0) * vic2;
        stressd1 = (stressd1 * vic1 + 2.0f * rmu * straind1) * vic2;
        stressd2 = (stressd2 * vic1 + 2.0f * rmu * straind2) * vic2;
        stress[0][1] = (stress[0][1] * vic1 + 2.0f * rmu * strain[0][1]) * vic2;
        stress[0][2] = (stress[0][2] * vic1 + 2.0f * rmu * strain[0][2]) * vic2;
        stress[1][2] = (stress[1][2] * vic1 + 2.0f * rmu * strain[1][2]) * vic2;
        VolumicStress = trace_stress / 3.0f + bulkm * trace_strain;
        stress[0][0] = stressd0 + VolumicStress;
        stress[1][1] = stressd1 + VolumicStress;
        stress[2][2] = stressd2 + VolumicStress;
    }
}

/* ---- Stress.c:53-172 ---------------------------------------------------------- */
static void stress_update(so_ctx* s, long e) {
    so_element* el = &s->el[e];
    const snac_material* m = &s->mat[el->material];
    double traceStress[NT], partialStress, sVolAvg, sOtherAvg;
    double phsDensity = m->density, alpha = m->alpha, beta = m->beta, pressure = 0.0f;
    double elemVolume = 2.0 * el->volume;
    for (int t = 0; t < NT; t++) {
        so_tet* tt = &el->tet[t];
        memset(tt->strain, 0, sizeof tt->strain);
        tt->strain[0][0] = tt->strainRate[0][0] * s->dt;
        tt->strain[1][1] = tt->strainRate[1][1] * s->dt;
        tt->strain[2][2] = tt->strainRate[2][2] * s->dt;
        tt->strain[0][1] = tt->strainRate[0][1] * s->dt;
        tt->strain[0][2] = tt->strainRate[0][2] * s->dt;
        tt->strain[1][2] = tt->strainRate[1][2] * s->dt;
    }
    /* Snac_EP_Constitutive: the one loaded constitutive plugin */
    switch (s->constitutive) {
        case SNAC_RHEOLOGY_ELASTIC: elastic_constitutive(s, e); break;
        case SNAC_RHEOLOGY_PLASTIC: plastic_constitutive(s, e); break;
        case SNAC_RHEOLOGY_VISCOPLASTIC: vp_constitutive(s, e); break;
        case SNAC_RHEOLOGY_MAXWELL: maxwell_constitutive(s, e); break;
        default: break;
    }
    partialStress = 0.0f;
    for (int t = 0; t < NT; t++) {
        so_tet* tt = &el->tet[t];
        for (int a = 0; a < 3; a++)
            for (int b = a; b < 3; b++)
                if (!isfinite(tt->stress[a][b])) fail(s, SNAC_GPU_ENAN, e, "stress is nan or inf");
        traceStress[t] = (tt->stress[0][0] + tt->stress[1][1] + tt->stress[2][2]) / 3.0f;
        partialStress += traceStress[t] * tt->volume;
    }
    sVolAvg = 0.0f;
    sOtherAvg = 0.0f;
    pressure = 0.0f;
    for (int t = 0; t < NT; t++) {
        double (*st)[3] = el->tet[t].stress;
        const double averageTraceStress = partialStress / elemVolume;
        st[0][0] += -1.0f * traceStress[t] + averageTraceStress;
        st[1][1] += -1.0f * traceStress[t] + averageTraceStress;
        st[2][2] += -1.0f * traceStress[t] + averageTraceStress;
        sVolAvg += (st[1][1] - averageTraceStress) * (st[2][2] - averageTraceStress) +
                   (st[2][2] - averageTraceStress) * (st[0][0] - averageTraceStress) +
                   (st[0][0] - averageTraceStress) * (st[1][1] - averageTraceStress);
        sOtherAvg += st[0][1] * st[0][1] + st[1][2] * st[1][2] + st[0][2] * st[0][2];
        pressure += (st[0][0] + st[1][1] + st[2][2]) / 3.0f;
    }
    sVolAvg /= NT;
    sOtherAvg /= NT;
    pressure /= NT;
    el->stress = 0.5f * sqrt(0.5f * fabs(-1.0f * sVolAvg + sOtherAvg));
    el->hydroPressure = -1.0 * pressure;
    if (!isfinite(el->stress)) fail(s, SNAC_GPU_ENAN, e, "element stress is nan or inf");
    for (int t = 0; t < NT; t++)
        el->tet[t].density = phsDensity * (1.0 - alpha * (el->tet[t].avgTemp - m->reftemp) + beta * pressure);
}

/* ---- Force.c:53-188 ------------------------------------------------------------ */
static void node_force(so_ctx* s, long n) {
    const double factor4 = 1.0f / 4.0f;
    const double gravity = s->gravity;
    double* f = s->force[n];
    double* bal = s->balance[n];
    double inertialMass = 0.0f, mass = 0.0f;
    long els[8];
    node_elements(s, n, els);
    f[0] = f[1] = f[2] = 0;
    bal[0] = bal[1] = bal[2] = 0;
    for (int ne = 0; ne < 8; ne++) {
        long e = els[ne];
        if (e < 0) continue;
        so_element* el = &s->el[e];
        const snac_material* m = &s->mat[el->material];
        const double inertialDensity = (m->lambda + 2.0f * m->mu) / (s->speedOfSound * s->speedOfSound);
        for (int idx = 0; idx < 5; idx++) {
            const so_tet* tt = &el->tet[NodeToTetra[ne][idx]];
            const double (*st)[3] = (const double (*)[3])tt->stress;
            const so_surface* surf = &tt->surface[NodeToSurface[ne][idx]];
            const double* nrm = surf->normal;
            const double effDensity = tt->density;
            if (s->dt_type == SNAC_DT_DYNAMIC) {
                inertialMass += factor4 * inertialDensity * tt->volume;
            } else if (s->dt_type == SNAC_DT_CONSTANT) {
                double alpha1 = (m->lambda + 2.0f * m->mu), temp, area_sum = 0.0;
                for (int d = 0; d < 3; d++) {
                    temp = (nrm[d] * surf->area) * (nrm[d] * surf->area);
                    if (temp > area_sum) area_sum = temp;
                }
                inertialMass += alpha1 * area_sum / (9.0f * tt->volume) * (s->dt * s->dt);
            } else {
                inertialMass += factor4 * effDensity * tt->volume;
            }
            f[0] += (st[0][0] * nrm[0] + st[0][1] * nrm[1] + st[0][2] * nrm[2]) * surf->area / 6.0f;
            f[1] += (st[0][1] * nrm[0] + st[1][1] * nrm[1] + st[1][2] * nrm[2]) * surf->area / 6.0f;
            f[2] += (st[0][2] * nrm[0] + st[1][2] * nrm[1] + st[2][2] * nrm[2]) * surf->area / 6.0f;
            f[1] -= gravity * effDensity * tt->volume / 8.0f;
            bal[0] += fabs(f[0]);
            bal[1] += fabs(f[1]);
            bal[2] += fabs(f[2]);
            mass += effDensity * tt->volume / 8.0;
        }
    }
    s->imass[n] = inertialMass;
    s->mass[n] = mass;
}

/* ---- tractionBC/Force.c:43-268: its active branch, a fixed stress on the right wall -- */
static void traction_force(so_ctx* s, long n) {
    const double factor4 = 1.0f / 4.0f;
    double* f = s->force[n];
    double* bal = s->balance[n];
    const long i = n % s->nnx;
    if (i != s->nnx - 1) return;
    double stress[3][3] = {{1.0e+08, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
    long els[8];
    node_elements(s, n, els);
    for (int ne = 0; ne < 8; ne++) {
        long e = els[ne];
        if (e < 0) continue;
        const double* c1 = s->coord[enode(s, e, 1)];
        const double* c2 = s->coord[enode(s, e, 2)];
        const double* c5 = s->coord[enode(s, e, 5)];
        const double* c6 = s->coord[enode(s, e, 6)];
        double n1[3], n2[3], normal[3];
        double area = so_tetrahedra_surface_area(c1, c2, c6) + so_tetrahedra_surface_area(c1, c6, c5);
        so_tetrahedra_surface_normal(c1, c2, c6, n1);
        so_tetrahedra_surface_normal(c1, c6, c5, n2);
        normal[0] = 0.5f * (n1[0] + n2[0]);
        normal[1] = 0.5f * (n1[1] + n2[1]);
        normal[2] = 0.5f * (n1[2] + n2[2]);
        f[0] += factor4 * area * (stress[0][0] * normal[0] + stress[0][1] * normal[1] + stress[0][2] * normal[2]);
        f[1] += factor4 * area * (stress[1][0] * normal[0] + stress[1][1] * normal[1] + stress[1][2] * normal[2]);
        f[2] += factor4 * area * (stress[2][0] * normal[0] + stress[2][1] * normal[1] + stress[2][2] * normal[2]);
        bal[0] += fabs(f[0]);
        bal[1] += fabs(f[1]);
        bal[2] += fabs(f[2]);
    }
}

/* ---- winkler/Force.c:56-168: bottom support (Winkler foundation) on j = 0 ---------- */
static void winkler_force(so_ctx* s, long n) {
    const double factor4 = 1.0f / 4.0f;
    double* f = s->force[n];
    const long j = (n / s->nnx) % s->nny;
    if (!(s->gravity > 0.0) || j != 0) return;
    long els[8];
    node_elements(s, n, els);
    const double nodeT = 0.0; /* the temperature lookup is compiled out (#if 0) */
    for (int ne = 0; ne < 8; ne++) {
        long e = els[ne];
        if (e < 0) continue;
        so_element* el = &s->el[e];
        const snac_material* m = &s->mat[el->material];
        const double phsDensity = m->density, drosub = 0.0f;
        double p_est = s->pisos + 0.5f * (phsDensity + drosub) * s->gravity * (s->coord[n][1] - s->rzbo);
        double rosubg = s->gravity * (phsDensity + drosub) * (1.0 - m->alpha * (nodeT - m->reftemp) + m->beta * p_est);
        double area = 0.0f, normal[3];
        double dhE = factor4 * (s->coord[enode(s, e, 0)][1] + s->coord[enode(s, e, 1)][1] +
                                s->coord[enode(s, e, 4)][1] + s->coord[enode(s, e, 5)][1]);
        const so_surface* s1 = &el->tet[1].surface[0];
        const so_surface* s2 = &el->tet[2].surface[1];
        const so_surface* s3 = &el->tet[6].surface[2];
        const so_surface* s4 = &el->tet[8].surface[2];
        area += s1->area;
        area += s2->area;
        area += s3->area;
        area += s4->area;
        normal[0] = factor4 * (s1->normal[0] + s2->normal[0] + s3->normal[0] + s4->normal[0]);
        normal[1] = -1.0f * factor4 * (s1->normal[1] + s2->normal[1] + s3->normal[1] + s4->normal[1]);
        normal[2] = factor4 * (s1->normal[2] + s2->normal[2] + s3->normal[2] + s4->normal[2]);
        area *= 0.5f;
        double press_norm = s->pisos + rosubg * (s->rzbo - dhE);
        f[0] += factor4 * (press_norm * area * normal[0]);
        f[1] += factor4 * (press_norm * area * normal[1]);
        f[2] += factor4 * (press_norm * area * normal[2]);
    }
    if (s->timeStep == 1) { /* restartTimestep == 0 */
        double Fy = f[1];
        if (Fy != 0.0) s->residualFr[n] = Fy;
    }
    f[1] -= s->residualFr[n];
}

#define getsign(val) ((val) < 0 ? -1.0f : (val) > 0 ? +1.0f : 0.0f)

/* ---- UpdateNode.c:161-857, cartesian: surface-topography diffusion ----------------
 * Run per node right after its coordinate update, in node order, so a top
 * node sees its -x and -z neighbours already updated (diffused, edge-copied)
 * and its +x and +z neighbours not yet moved this step. */
static int top_interior(const so_ctx* s, long i, long k) { return i > 0 && i < s->nnx - 1 && k > 0 && k < s->nnz - 1; }

/* :161-260 */
static void get_max_topo_grad(so_ctx* s, long n) {
    const long i = n % s->nnx, j = (n / s->nnx) % s->nny, k = n / ((long)s->nnx * s->nny);
    if (s->timeStep <= 1 || j < s->nny - 1 || !top_interior(s, i, k)) return;
    const double* X0 = s->coord[n];
    const double* xR = s->coord[n + 1];
    const double* xF = s->coord[n + (long)s->nnx * s->nny];
    double dydx = (xR[1] - X0[1]) / (xR[0] - X0[0]);
    double dydz = (xF[1] - X0[1]) / (xF[2] - X0[2]);
    double localTopoGrad = sqrt(dydx * dydx + dydz * dydz);
    s->topoGradMax = (s->topoGradMax > localTopoGrad) ? s->topoGradMax : localTopoGrad;
}

/* :359-506 and :647-715 (DiffTopo, UpdateInteriorTopo) */
static void diff_topo(so_ctx* s, long n) {
    const long i = n % s->nnx, j = (n / s->nnx) % s->nny, k = n / ((long)s->nnx * s->nny);
    if (s->timeStep <= 1 || j < s->nny - 1 || s->topoGradMax < s->topoGradCriterion) return;
    if (!top_interior(s, i, k)) return;
    const long sz = (long)s->nnx * s->nny;
    double* X0 = s->coord[n];
    const double *xR = s->coord[n + 1], *xL = s->coord[n - 1], *xF = s->coord[n + sz], *xB = s->coord[n - sz];
    double dydx1 = (xR[1] - X0[1]) / (xR[0] - X0[0]);
    double dydx2 = (X0[1] - xL[1]) / (X0[0] - xL[0]);
    double d2ydx2 = (dydx1 - dydx2) / (0.5f * (xR[0] - xL[0]));
    double dydz1 = (xF[1] - X0[1]) / (xF[2] - X0[2]);
    double dydz2 = (X0[1] - xB[1]) / (X0[2] - xB[2]);
    double d2ydz2 = (dydz1 - dydz2) / (0.5f * (xF[2] - xB[2]));
    double lapl_topo = d2ydx2 + d2ydz2;
    double dh = s->topo_kappa * s->dt * lapl_topo;
    X0[1] += dh;
}

/* :716-857 (AdjustEdgeTopo) */
static void adjust_edge_topo(so_ctx* s, long n) {
    const long i = n % s->nnx, j = (n / s->nnx) % s->nny, k = n / ((long)s->nnx * s->nny);
    if (s->timeStep <= 1 || j < s->nny - 1 || s->topoGradMax < s->topoGradCriterion) return;
    const long sz = (long)s->nnx * s->nny;
    const double *xN1 = NULL, *xN2 = NULL;
    if (i == 0) xN1 = s->coord[n + 1];
    else if (i == s->nnx - 1) xN1 = s->coord[n - 1];
    if (k == 0) xN2 = s->coord[n + sz];
    else if (k == s->nnz - 1) xN2 = s->coord[n - sz];
    double* X0 = s->coord[n];
    if (xN1 && !xN2) X0[1] = xN1[1];
    else if (!xN1 && xN2) X0[1] = xN2[1];
    else if (xN1 && xN2) X0[1] = 0.5f * (xN1[1] + xN2[1]);
}

/* ---- UpdateNode.c:74-158 (PreProcess) then :60-72 ------------------------------ */
static void node_update(so_ctx* s, long n) {
    double* v = s->vel[n];
    double* f = s->force[n];
    double m = s->imass[n];
    f[0] -= s->demf * getsign(v[0]) * fabs(f[0]);
    f[1] -= s->demf * getsign(v[1]) * fabs(f[1]);
    f[2] -= s->demf * getsign(v[2]) * fabs(f[2]);
    if (!isfinite(f[0]) || !isfinite(f[1]) || !isfinite(f[2])) fail(s, SNAC_GPU_ENAN, n, "force is nan or inf");
    v[0] += s->dt * f[0] / m;
    v[1] += s->dt * f[1] / m;
    v[2] += s->dt * f[2] / m;
    /* VariableCondition_ApplyToIndex with last-VC-wins values */
    unsigned char mask = s->vbc_mask[n];
    for (int d = 0; d < 3; d++)
        if (mask & (1u << d)) v[d] = s->vbc_val[n][d];
    double* c = s->coord[n];
    c[0] += s->dt * v[0];
    c[1] += s->dt * v[1];
    c[2] += s->dt * v[2];
    if (s->topo_kappa > 0) get_max_topo_grad(s, n);
    /* the topography hooks appended after UpdateNodeMomentum, Context.c:578-592 */
    diff_topo(s, n);
    adjust_edge_topo(s, n);
}

/* ---- temperature/HeatFlux.c:60-200 --------------------------------------------- */
static void heat_flux(so_ctx* s, long e) {
    so_element* el = &s->el[e];
    const snac_material* m = &s->mat[el->material];
    const double bulkm = m->lambda + 2.0f * m->mu / 3.0f;
    const double alpha = m->alpha;
    double temp = 0.0f, temp0 = 0.0f;
    for (int t = 0; t < NT; t++) {
        so_tet* tt = &el->tet[t];
        double T[4], T0v[4];
        for (int q = 0; q < 4; q++) {
            long nn = enode(s, e, TetraToNode[t][q]);
            T[q] = s->T[nn];
            T0v[q] = s->T0[nn];
        }
        const so_surface* S = tt->surface;
        for (int d = 0; d < 3; d++)
            tt->heatFlux[d] = 1.0f * m->thermal_conduct *
                              (T[0] * S[1].normal[d] * S[1].area + T[1] * S[2].normal[d] * S[2].area +
                               T[2] * S[3].normal[d] * S[3].area + T[3] * S[0].normal[d] * S[0].area) /
                              3.0f / tt->volume;
        if (s->thermal_stress) {
            temp = 0.25f * (T[0] + T[1] + T[2] + T[3]);
            temp0 = 0.25f * (T0v[0] + T0v[1] + T0v[2] + T0v[3]);
            tt->thermalStress = -1.0f * alpha * bulkm * (temp - temp0);
        }
    }
}

/* temperature/VariableConditions.c:280-413 */
static void heat_flux_bc(so_ctx* s) {
    for (long e = 0; e < s->ne; e++) {
        int ei = (int)(e % s->nx), ek = (int)(e / ((long)s->nx * s->ny));
        so_element* el = &s->el[e];
        double g[4], Fn, normal[3] = {0, 0, 0};
        if (!(ei == 0 || ei == s->nx - 1 || ek == 0 || ek == s->nz - 1)) continue;
#define NSUM4(t0, f0, t1, f1, t2, f2, t3, f3, d)                                                  \
    (0.25f * (el->tet[t0].surface[f0].normal[d] + el->tet[t1].surface[f1].normal[d] +            \
              el->tet[t2].surface[f2].normal[d] + el->tet[t3].surface[f3].normal[d]))
        if (ei == 0)
            for (int d = 0; d < 3; d++) normal[d] = NSUM4(0, 2, 1, 2, 5, 0, 6, 0, d);
        if (ei == s->nx - 1)
            for (int d = 0; d < 3; d++) normal[d] = NSUM4(2, 0, 3, 0, 7, 0, 8, 0, d);
        if (ek == 0)
            for (int d = 0; d < 3; d++) normal[d] = NSUM4(0, 1, 2, 2, 6, 1, 7, 1, d);
        if (ek == s->nz - 1)
            for (int d = 0; d < 3; d++) normal[d] = NSUM4(1, 1, 3, 2, 5, 1, 8, 1, d);
#undef NSUM4
        for (int t = 0; t < NT; t++) {
            so_tet* tt = &el->tet[t];
            const so_surface* S = tt->surface;
            double T[4];
            for (int q = 0; q < 4; q++) T[q] = s->T[enode(s, e, TetraToNode[t][q])];
            for (int d = 0; d < 3; d++)
                g[d] = -1.0f *
                       (T[0] * S[1].normal[d] * S[1].area + T[1] * S[2].normal[d] * S[2].area +
                        T[2] * S[3].normal[d] * S[3].area + T[3] * S[0].normal[d] * S[0].area) /
                       3.0f / tt->volume;
            Fn = 0.0f;
            for (int i = 0; i < 3; i++) Fn += g[i] * normal[i];
            tt->heatFlux[0] -= Fn * normal[0];
            tt->heatFlux[1] -= Fn * normal[1];
            tt->heatFlux[2] -= Fn * normal[2];
        }
    }
}

/* temperature/Heat.c:64-140 with sourceterm = 0 */
static void node_heat(so_ctx* s, long n, double* newT) {
    double energy = 0.0f, source = 0.0f, lumpVolume = 0.0f, sourceterm = 0.0;
    long els[8];
    node_elements(s, n, els);
    for (int ne = 0; ne < 8; ne++) {
        long e = els[ne];
        if (e < 0) continue;
        so_element* el = &s->el[e];
        const snac_material* m = &s->mat[el->material];
        for (int idx = 0; idx < 5; idx++) {
            const so_tet* tt = &el->tet[NodeToTetra[ne][idx]];
            const double* hf = tt->heatFlux;
            const so_surface* surf = &tt->surface[NodeToSurface[ne][idx]];
            const double* nrm = surf->normal;
            energy += (hf[0] * nrm[0] + hf[1] * nrm[1] + hf[2] * nrm[2]) * surf->area / 6.0f;
            source += sourceterm * tt->volume / 4.0f;
            lumpVolume += m->heat_capacity *
                          (((tt->density == 0.0)
                                ? (m->density * (1.0 - m->alpha * (tt->avgTemp - m->reftemp) + m->beta * el->hydroPressure))
                                : tt->density) *
                           tt->volume) /
                          8.0f;
        }
        double dt_thermal_to_mech = sqrt((m->lambda + 2.0f * m->mu) / m->density) * s->minLengthScale /
                                    (m->thermal_conduct / (m->heat_capacity * m->density));
        if (!(dt_thermal_to_mech > 1.0)) fail(s, SNAC_GPU_EPHYSICS, n, "dt_thermal/dt_mech <= 1");
    }
    newT[0] = s->T[n];
    newT[1] = s->T[n] + (energy + source) * -1.0f * s->dt / lumpVolume;
}

static void apply_temperature_bcs(so_ctx* s) {
    for (long n = 0; n < s->nn; n++)
        if (s->tbc_mask[n]) s->T[n] = s->tbc_val[n];
}

/* ---- loop drivers (Context.c:1063-1184, Heat.c:47-62, HeatFlux.c:47-58) ------- */
int so_loop_elements_energy(so_ctx* s) {
    if (!s->temperature) return 0;
    for (long e = 0; e < s->ne; e++) heat_flux(s, e);
    heat_flux_bc(s);
    return s->status;
}

int so_loop_nodes_energy(so_ctx* s) {
    if (!s->temperature) return 0;
    /* nodes are updated in index order; Snac_Heat reads no other node's T */
    double nt[2];
    for (long n = 0; n < s->nn; n++) {
        node_heat(s, n, nt);
        s->T0[n] = nt[0];
        s->T[n] = nt[1];
    }
    /* UpdateAverageTemp_LoopElements, Heat.c:143-172 */
    for (long e = 0; e < s->ne; e++)
        for (int t = 0; t < NT; t++) {
            so_tet* tt = &s->el[e].tet[t];
            tt->avgTemp = 0.0;
            for (int q = 0; q < 4; q++) tt->avgTemp += s->T[enode(s, e, TetraToNode[t][q])] / (1.0f * 4);
        }
    apply_temperature_bcs(s);
    return s->status;
}

int so_calc_stresses(so_ctx* s) {
    for (long e = 0; e < s->ne; e++) {
        strain_rate(s, e);
        stress_update(s, e);
    }
    return s->status;
}

/* Snac_Force for every node without the node update (the force loop of
 * _Snac_Context_LoopNodes, Context.c:1129-1140) */
int so_node_forces(so_ctx* s) {
    for (long n = 0; n < s->nn; n++) {
        node_force(s, n);
        if (s->winkler) winkler_force(s, n); /* appended to Snac_EP_Force, winkler/Register.c:140-145 */
        if (s->traction) traction_force(s, n); /* tractionBC/Register.c:79-83 */
    }
    return s->status;
}

int so_loop_nodes_momentum(so_ctx* s) {
    for (long n = 0; n < s->nn; n++) {
        node_force(s, n);
        if (s->winkler) winkler_force(s, n); /* appended to Snac_EP_Force, winkler/Register.c:140-145 */
        if (s->traction) traction_force(s, n); /* tractionBC/Register.c:79-83 */
    }
    for (long n = 0; n < s->nn; n++) node_update(s, n);
    return s->status;
}

int so_loop_elements_momentum(so_ctx* s) {
    update_element(s, 0, &s->minLengthScale);
    for (long e = 1; e < s->ne; e++) {
        double ls;
        update_element(s, e, &ls);
        if (ls < s->minLengthScale) s->minLengthScale = ls;
    }
    return s->status;
}

/* _Snac_Context_Sync, Context.c:1208-1268 */
int so_sync(so_ctx* s) {
    double v, vx, vy, vz, vmax = 0.0f, vlb = 3.0e-11f;
    for (long q = 0; q < s->n_vbc_nodes; q++) {
        long n = s->vbc_nodes[q];
        vx = s->vel[n][0];
        vy = s->vel[n][1];
        vz = s->vel[n][2];
        v = sqrt(vx * vx + vy * vy + vz * vz);
        if (v > vmax) vmax = v;
    }
    if (vmax < vlb) vmax = vlb;
    s->vmax = vmax;
    if (s->timeStep == 0) s->initMinLengthScale = s->minLengthScale;
    if (s->dt_type == SNAC_DT_DYNAMIC) {
        s->dt = s->minLengthScale * 0.45f * s->strain_inert / vmax;
        s->speedOfSound = s->minLengthScale * 0.5f / s->dt;
    } else if (s->dt_type == SNAC_DT_WAVE) {
        s->dt = 0.5f * s->minLengthScale / s->speedOfSound;
    }
    return s->status;
}

/* Snac_Context_TimeStepZero, Context.c:978-1036 (not restarting) */
int so_time_step_zero(so_ctx* s) {
    for (long e = 0; e < s->ne; e++) {
        so_element* el = &s->el[e];
        double phsDensity = s->mat[el->material].density, sVolAvg = 0.0f;
        el->stress = 0;
        for (int t = 0; t < NT; t++) {
            double (*st)[3] = el->tet[t].stress;
            sVolAvg += st[1][1] * st[2][2] + st[2][2] * st[0][0] + st[0][0] * st[1][1];
            el->tet[t].avgTemp = 0.0f;
            el->tet[t].density = phsDensity;
        }
        el->stress = 0.5f * sqrt(0.5f * fabs(sVolAvg / NT));
    }
    so_loop_elements_momentum(s);
    so_sync(s);
    return s->status;
}

/* _AbstractContext_Execute_Hook / _AbstractContext_Step, AbstractContext.c:874-941 */
int so_begin_step(so_ctx* s) {
    s->timeStep++;
    s->dt = 1.0 * s->dt; /* dtFactor * AbstractContext_Dt */
    s->currentTime += s->dt;
    return s->status;
}

int so_step(so_ctx* s, int nsteps) {
    for (int i = 0; i < nsteps && s->status == 0; i++) {
        so_begin_step(s);
        so_loop_elements_energy(s);
        so_loop_nodes_energy(s);
        so_calc_stresses(s);
        so_loop_nodes_momentum(s);
        so_loop_elements_momentum(s);
        so_sync(s);
    }
    return s->status;
}

/* ---- construction and initial conditions ---------------------------------------- */
static int wall_has(const so_ctx* s, int wall, int i, int j, int k) {
    switch (wall) {
        case SNAC_WALL_BACK: return k == 0;
        case SNAC_WALL_LEFT: return i == 0;
        case SNAC_WALL_BOTTOM: return j == 0;
        case SNAC_WALL_RIGHT: return i == s->nnx - 1;
        case SNAC_WALL_TOP: return j == s->nny - 1;
        case SNAC_WALL_FRONT: return k == s->nnz - 1;
        case SNAC_WALL_ALL: return 1;
        default: return 0;
    }
}

/* hydroStaticIC/VariableConditions.c:43-152, one rank */
static void hydrostatic_ic(so_ctx* s, double ymin) {
    s->rzbo = ymin; /* element->rzbo = geometry->min[1], :120 */
    for (int elK = 0; elK < s->nz; elK++)
        for (int elI = 0; elI < s->nx; elI++) {
            double rogh = 0.0f;
            for (int elJ = s->ny - 1; elJ > -1; elJ--) {
                long e = elI + (long)elJ * s->nx + (long)elK * s->nx * s->ny;
                so_element* el = &s->el[e];
                const snac_material* m = &s->mat[el->material];
                double phsDensity = m->density, alpha = m->alpha, beta = m->beta, densT = 0.0f;
                double dhE[4], dh, dPT, dP, P;
                for (int t = 0; t < NT; t++) {
                    so_tet* tt = &el->tet[t];
                    densT += ((tt->density == 0.0) ? (phsDensity * (1.0 - alpha * (tt->avgTemp - m->reftemp)))
                                                   : (tt->density)) /
                             NT;
                    memset(tt->strainRate, 0, sizeof tt->strainRate);
                }
                dhE[0] = s->coord[enode(s, e, 6)][1] - s->coord[enode(s, e, 0)][1];
                dhE[1] = s->coord[enode(s, e, 2)][1] - s->coord[enode(s, e, 4)][1];
                dhE[2] = s->coord[enode(s, e, 3)][1] - s->coord[enode(s, e, 5)][1];
                dhE[3] = s->coord[enode(s, e, 7)][1] - s->coord[enode(s, e, 1)][1];
                dh = 0.25f * (dhE[0] + dhE[1] + dhE[2] + dhE[3]);
                el->stress = 0.0;
                el->strainRate = 0.0;
                el->hydroPressure = 0.0f;
                dPT = densT * s->gravity * dh;
                dP = dPT * (1.0 - beta * rogh) / (1.0f + beta / 2.0f * dPT);
                P = rogh + 0.5f * dP;
                P = -1.0f * (P + 0.0);
                for (int t = 0; t < NT; t++) {
                    el->tet[t].stress[0][0] = P;
                    el->tet[t].stress[1][1] = P;
                    el->tet[t].stress[2][2] = P;
                }
                el->hydroPressure = P;
                rogh += dP;
                /* the isostatic pressure at the bottom of column (0, 0), :133-140 */
                if (elJ == 0 && elI == 0 && elK == 0) s->pisos = rogh + 0.0;
            }
        }
}

so_ctx* so_create(const snac_gpu_desc* d, int* status) {
    *status = SNAC_GPU_EINVAL;
    if (!d || d->nx < 1 || d->ny < 1 || d->nz < 1 || d->n_materials < 1 || !d->materials) return NULL;
    so_ctx* s = (so_ctx*)calloc(1, sizeof *s);
    s->nx = d->nx;
    s->ny = d->ny;
    s->nz = d->nz;
    s->nnx = d->nx + 1;
    s->nny = d->ny + 1;
    s->nnz = d->nz + 1;
    s->ne = (long)d->nx * d->ny * d->nz;
    s->nn = (long)s->nnx * s->nny * s->nnz;
    s->dt_type = d->dt_type;
    s->dt = d->dt;
    s->strain_inert = d->strain_inert;
    s->gravity = d->gravity;
    s->demf = d->demf;
    s->constitutive = d->constitutive;
    s->temperature = d->temperature;
    s->thermal_stress = d->compute_thermal_stress;
    s->speedOfSound = 0.0f;
    s->minLengthScale = 0.0f;
    s->err_index = -1;
    s->coord = calloc(s->nn, sizeof *s->coord);
    s->vel = calloc(s->nn, sizeof *s->vel);
    s->force = calloc(s->nn, sizeof *s->force);
    s->balance = calloc(s->nn, sizeof *s->balance);
    s->imass = calloc(s->nn, sizeof(double));
    s->winkler = d->winkler;
    s->traction = d->traction_bc;
    s->topo_kappa = d->topo_kappa;
    s->topoGradCriterion = d->topo_grad_criterion;
    s->topoGradMax = 0.0f;
    if (s->topo_kappa > 0 && (s->nnx <= 2 || s->nnz <= 2)) {
        free(s);
        *status = SNAC_GPU_ENOTSUP; /* the one-element-wide variants are not restated */
        return NULL;
    }
    s->residualFr = calloc(s->nn, sizeof(double));
    s->mass = calloc(s->nn, sizeof(double));
    s->T = calloc(s->nn, sizeof(double));
    s->T0 = calloc(s->nn, sizeof(double));
    s->el = calloc(s->ne, sizeof(so_element));
    s->vbc_mask = calloc(s->nn, 1);
    s->vbc_val = calloc(s->nn, sizeof *s->vbc_val);
    s->vbc_nodes = calloc(s->nn, sizeof(long));
    s->tbc_mask = calloc(s->nn, 1);
    s->tbc_val = calloc(s->nn, sizeof(double));
    if (!s->coord || !s->vel || !s->el || !s->tbc_val) {
        *status = SNAC_GPU_ENOMEM;
        so_destroy(s);
        return NULL;
    }
    /* Phases.  Per-element table multipliers are expressed, as the reference
     * would see them, as one phase per element with scaled table values. */
    int per_elem = d->element_cohesion_scale || d->element_friction_scale || d->element_visc_scale;
    if (per_elem && d->constitutive == SNAC_RHEOLOGY_MAXWELL) {
        /* the Maxwell hook only flags phase 0 (maxwell/InitialConditions.c:53) */
        *status = SNAC_GPU_ENOTSUP;
        so_destroy(s);
        return NULL;
    }
    s->nmat = per_elem ? (int)s->ne : d->n_materials;
    s->mat = calloc(s->nmat, sizeof(snac_material));
    s->rheology = calloc(s->nmat, sizeof(unsigned));
    for (long e = 0; e < s->ne; e++) {
        int m = d->element_material ? d->element_material[e] : 0;
        if (m < 0 || m >= d->n_materials) {
            *status = SNAC_GPU_EMATERIAL;
            so_destroy(s);
            return NULL;
        }
        if (per_elem) {
            snac_material mm = d->materials[m];
            for (int i = 0; i <= SNAC_MAX_SEGMENTS; i++) {
                if (d->element_cohesion_scale) mm.cohesion[i] = mm.cohesion[i] * d->element_cohesion_scale[e];
                if (d->element_friction_scale)
                    mm.friction_angle[i] = mm.friction_angle[i] * d->element_friction_scale[e];
            }
            if (d->element_visc_scale) mm.refvisc = mm.refvisc * d->element_visc_scale[e];
            s->mat[e] = mm;
            s->el[e].material = (int)e;
        } else {
            s->el[e].material = m;
        }
    }
    if (!per_elem)
        for (int m = 0; m < d->n_materials; m++) s->mat[m] = d->materials[m];
    /* Drucker-Prager iteration controls of each phase (defaults 1 and 1e-3) */
    s->maxiterations = calloc(s->nmat, sizeof(int));
    s->tolerance = calloc(s->nmat, sizeof(double));
    for (int p = 0; p < s->nmat; p++) {
        int src = per_elem ? (d->element_material ? d->element_material[p] : 0) : p;
        s->maxiterations[p] = d->dp_max_iterations ? d->dp_max_iterations[src] : 1;
        s->tolerance[p] = d->dp_tolerance ? d->dp_tolerance[src] : 1.e-3;
    }
    /* rheology is hard-wired to Elastic (Context.c:834); the plugin ICs OR in
     * their bit (plastic/InitialConditions.c:57, viscoplastic/InitialConditions.c:64,
     * maxwell/InitialConditions.c:53 - phase 0 only) */
    for (int m = 0; m < s->nmat; m++) {
        s->rheology[m] = SNAC_RHEOLOGY_ELASTIC;
        if (d->constitutive == SNAC_RHEOLOGY_PLASTIC) s->rheology[m] |= SNAC_RHEOLOGY_PLASTIC;
        if (d->constitutive == SNAC_RHEOLOGY_VISCOPLASTIC) s->rheology[m] |= SNAC_RHEOLOGY_VISCOPLASTIC;
    }
    if (d->constitutive == SNAC_RHEOLOGY_MAXWELL)
        for (int m = 0; m < s->nmat; m++)
            if (per_elem || m == 0) s->rheology[m] |= SNAC_RHEOLOGY_MAXWELL;
    /* mesh coordinates: BlockGeometry.c:326-349 */
    for (long n = 0; n < s->nn; n++) {
        int i = (int)(n % s->nnx), j = (int)((n / s->nnx) % s->nny), k = (int)(n / ((long)s->nnx * s->nny));
        if (d->node_coords) {
            for (int q = 0; q < 3; q++) s->coord[n][q] = d->node_coords[n * 3 + q];
        } else {
            int ijk[3] = {i, j, k}, size[3] = {s->nnx, s->nny, s->nnz};
            for (int q = 0; q < 3; q++)
                s->coord[n][q] = size[q] > 1 ? d->min[q] + (d->max[q] - d->min[q]) * ((double)ijk[q] / (double)(size[q] - 1))
                                             : d->min[q];
        }
        /* nodeICs */
        if (d->init_velocity)
            for (int q = 0; q < 3; q++) s->vel[n][q] = d->init_velocity[n * 3 + q];
        if (d->temperature) {
            if (d->temperature_sweep_ic)
                /* _SnacTemperature_Top2BottomSweep, temperature/VariableConditions.c:52-73 */
                s->T[n] = d->bottom_temp + (d->top_temp - d->bottom_temp) / (s->nny - 1) * j;
            else if (d->init_temperature)
                s->T[n] = d->init_temperature[n];
        }
        /* velocity BCs: union of wall sets, last VC wins per component */
        for (int b = 0; b < d->n_velocity_bcs; b++) {
            const snac_wall_bc* bc = &d->velocity_bcs[b];
            if (!wall_has(s, bc->wall, i, j, k)) continue;
            for (int q = 0; q < 3; q++)
                if (bc->mask & (1 << q)) {
                    s->vbc_mask[n] |= (unsigned char)(1u << q);
                    s->vbc_val[n][q] = bc->value[q];
                }
        }
        if (s->vbc_mask[n]) s->vbc_nodes[s->n_vbc_nodes++] = n;
        for (int b = 0; b < d->n_temperature_bcs; b++) {
            const snac_wall_bc* bc = &d->temperature_bcs[b];
            if (!wall_has(s, bc->wall, i, j, k) || !(bc->mask & 1)) continue;
            s->tbc_mask[n] = 1;
            s->tbc_val[n] = bc->value[0];
        }
    }
    /* elementICs: stress */
    if (d->init_stress)
        for (long e = 0; e < s->ne; e++)
            for (int t = 0; t < NT; t++) {
                const double* q = &d->init_stress[(e * NT + t) * 6];
                double (*st)[3] = s->el[e].tet[t].stress;
                st[0][0] = q[0];
                st[1][1] = q[1];
                st[2][2] = q[2];
                st[0][1] = q[3];
                st[0][2] = q[4];
                st[1][2] = q[5];
            }
    /* VariableCondition_Apply(velocityBCs), Context.c:773 */
    for (long n = 0; n < s->nn; n++)
        for (int q = 0; q < 3; q++)
            if (s->vbc_mask[n] & (1u << q)) s->vel[n][q] = s->vbc_val[n][q];
    /* plugin ICs before SnacTimeStepZero */
    if (d->temperature) {
        for (long n = 0; n < s->nn; n++) s->T0[n] = s->T[n];
        apply_temperature_bcs(s);
    }
    if (d->constitutive == SNAC_RHEOLOGY_VISCOPLASTIC) {
        for (long e = 0; e < s->ne; e++)
            for (int t = 0; t < NT; t++) s->el[e].tet[t].viscosity = s->mat[s->el[e].material].vis_min;
        /* viscoplastic/InitialConditions.c:84-90: dt = min(dt, 0.9 vis_min/mu) */
        double dtm = 0;
        for (int m = 0; m < (per_elem ? 1 : s->nmat); m++) {
            double v = 9.0e-01 * s->mat[m].vis_min / s->mat[m].mu;
            dtm = (m == 0) ? v : (v < dtm ? v : dtm);
        }
        if (s->dt > dtm && s->dt_type != SNAC_DT_CONSTANT) s->dt = dtm;
    }
    if (d->constitutive == SNAC_RHEOLOGY_MAXWELL) {
        /* maxwell/InitialConditions.c:55-66: a constant dt above the bound hits
         * assert(0), which the -DNDEBUG reference build compiles out */
        double dtm = 1.0e-01 * s->mat[0].vis_min / s->mat[0].mu;
        if (s->dt > dtm && s->dt_type != SNAC_DT_CONSTANT) s->dt = dtm;
    }
    if (d->hydrostatic_ic) hydrostatic_ic(s, d->min[1]);
    s->timeStep = 0;
    *status = 0;
    return s;
}

void so_destroy(so_ctx* s) {
    if (!s) return;
    free(s->coord);
    free(s->vel);
    free(s->force);
    free(s->balance);
    free(s->imass);
    free(s->residualFr);
    free(s->mass);
    free(s->T);
    free(s->T0);
    free(s->el);
    free(s->vbc_mask);
    free(s->vbc_val);
    free(s->vbc_nodes);
    free(s->tbc_mask);
    free(s->tbc_val);
    free(s->mat);
    free(s->rheology);
    free(s->maxiterations);
    free(s->tolerance);
    free(s);
}

/* ---- state access ------------------------------------------------------------------ */
int so_get_state(so_ctx* s, const snac_state_view* v) {
    for (long n = 0; n < s->nn; n++)
        for (int q = 0; q < 3; q++) {
            if (v->coord) v->coord[n * 3 + q] = s->coord[n][q];
            if (v->velocity) v->velocity[n * 3 + q] = s->vel[n][q];
            if (v->force) v->force[n * 3 + q] = s->force[n][q];
        }
    for (long n = 0; n < s->nn; n++) {
        if (v->temperature) v->temperature[n] = s->T[n];
        if (v->inertial_mass) v->inertial_mass[n] = s->imass[n];
    }
    for (long e = 0; e < s->ne; e++)
        for (int t = 0; t < NT; t++) {
            const so_tet* tt = &s->el[e].tet[t];
            if (v->stress) {
                double* q = &v->stress[(e * NT + t) * 6];
                q[0] = tt->stress[0][0];
                q[1] = tt->stress[1][1];
                q[2] = tt->stress[2][2];
                q[3] = tt->stress[0][1];
                q[4] = tt->stress[0][2];
                q[5] = tt->stress[1][2];
            }
            if (v->plastic_strain) v->plastic_strain[e * NT + t] = tt->plasticStrain;
            if (v->viscosity) v->viscosity[e * NT + t] = tt->viscosity;
            if (v->plastic_strain_tensor) {
                double* q = &v->plastic_strain_tensor[(e * NT + t) * 6];
                q[0] = tt->plasticstrainTensor[0][0];
                q[1] = tt->plasticstrainTensor[1][1];
                q[2] = tt->plasticstrainTensor[2][2];
                q[3] = tt->plasticstrainTensor[0][1];
                q[4] = tt->plasticstrainTensor[0][2];
                q[5] = tt->plasticstrainTensor[1][2];
            }
        }
    return 0;
}

int so_set_state(so_ctx* s, const snac_state_view* v) {
    for (long n = 0; n < s->nn; n++)
        for (int q = 0; q < 3; q++) {
            if (v->coord) s->coord[n][q] = v->coord[n * 3 + q];
            if (v->velocity) s->vel[n][q] = v->velocity[n * 3 + q];
        }
    for (long n = 0; n < s->nn; n++)
        if (v->temperature) s->T[n] = v->temperature[n];
    for (long e = 0; e < s->ne; e++)
        for (int t = 0; t < NT; t++) {
            so_tet* tt = &s->el[e].tet[t];
            if (v->stress) {
                const double* q = &v->stress[(e * NT + t) * 6];
                tt->stress[0][0] = q[0];
                tt->stress[1][1] = q[1];
                tt->stress[2][2] = q[2];
                tt->stress[0][1] = q[3];
                tt->stress[0][2] = q[4];
                tt->stress[1][2] = q[5];
            }
            if (v->plastic_strain) tt->plasticStrain = v->plastic_strain[e * NT + t];
            if (v->viscosity) tt->viscosity = v->viscosity[e * NT + t];
            if (v->plastic_strain_tensor) {
                const double* q = &v->plastic_strain_tensor[(e * NT + t) * 6];
                tt->plasticstrainTensor[0][0] = q[0];
                tt->plasticstrainTensor[1][1] = q[1];
                tt->plasticstrainTensor[2][2] = q[2];
                tt->plasticstrainTensor[0][1] = q[3];
                tt->plasticstrainTensor[0][2] = q[4];
                tt->plasticstrainTensor[1][2] = q[5];
            }
        }
    return 0;
}

void so_scalars(so_ctx* s, snac_scalars* o) {
    o->dt = s->dt;
    o->min_length_scale = s->minLengthScale;
    o->vmax = s->vmax;
    o->speed_of_sound = s->speedOfSound;
    o->time_step = s->timeStep;
    o->current_time = s->currentTime;
}

void so_set_dt(so_ctx* s, double dt) { s->dt = dt; }

const char* so_last_error(so_ctx* s) { return s->status ? s->err : ""; }

void so_get_geometry(so_ctx* s, double* volume, double* area, double* normal) {
    for (long e = 0; e < s->ne; e++)
        for (int t = 0; t < NT; t++) {
            const so_tet* tt = &s->el[e].tet[t];
            if (volume) volume[e * NT + t] = tt->volume;
            for (int f = 0; f < 4; f++) {
                if (area) area[(e * NT + t) * 4 + f] = tt->surface[f].area;
                if (normal)
                    for (int q = 0; q < 3; q++) normal[((e * NT + t) * 4 + f) * 3 + q] = tt->surface[f].normal[q];
            }
        }
}

void so_get_element_scalars(so_ctx* s, double* volume, double* strain_rate, double* stress,
                            double* hydro_pressure, double* aps, double* min_length_scale) {
    for (long e = 0; e < s->ne; e++) {
        const so_element* el = &s->el[e];
        if (volume) volume[e] = el->volume;
        if (strain_rate) strain_rate[e] = el->strainRate;
        if (stress) stress[e] = el->stress;
        if (hydro_pressure) hydro_pressure[e] = el->hydroPressure;
        if (aps) aps[e] = el->aps;
        if (min_length_scale) min_length_scale[e] = el->minLengthScale;
    }
}

void so_get_tet_fields(so_ctx* s, double* strain_rate, double* strain, double* density, double* avg_temp) {
    static const int ia[6] = {0, 1, 2, 0, 0, 1}, ib[6] = {0, 1, 2, 1, 2, 2};
    for (long e = 0; e < s->ne; e++)
        for (int t = 0; t < NT; t++) {
            const so_tet* tt = &s->el[e].tet[t];
            for (int c = 0; c < 6; c++) {
                if (strain_rate) strain_rate[(e * NT + t) * 6 + c] = tt->strainRate[ia[c]][ib[c]];
                if (strain) strain[(e * NT + t) * 6 + c] = tt->strain[ia[c]][ib[c]];
            }
            if (density) density[e * NT + t] = tt->density;
            if (avg_temp) avg_temp[e * NT + t] = tt->avgTemp;
        }
}

void so_get_node_fields(so_ctx* s, double* mass, double* balance) {
    for (long n = 0; n < s->nn; n++) {
        if (mass) mass[n] = s->mass[n];
        if (balance)
            for (int q = 0; q < 3; q++) balance[n * 3 + q] = s->balance[n][q];
    }
}
