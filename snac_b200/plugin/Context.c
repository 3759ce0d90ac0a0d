/*
 * Context.c — between a Snac_Context and the device model: which plugins the
 * context carries, the descriptor built from it, and the state copied between
 * its arrays of structs and the library's element-major arrays.
 *
 * The context's layout is the reference's: nodes through Snac_Node_At (the
 * node array with its extensions, Snac/libSnac/src/shortcuts.h:47-48,
 * Node.h:47-58), coordinates in mesh->nodeCoord, per-tet state in
 * Snac_Element::tetra[10] (Element.h:45-77), and the plugins' data in their
 * extensions, found by key (ExtensionManager_GetHandle,
 * StGermain/Base/Extensibility/src/ExtensionManager.c:678-699): SnacPlastic,
 * SnacViscoPlastic, SnacMaxwell element extensions (plastic strain,
 * viscosity), the SnacTemperature node and context extensions.
 */
#include <mpi.h>
#include <StGermain/StGermain.h>
#include <StGermain/FD/FD.h>
#include "Snac/Snac.h"
#include "Snac/Plastic/Plastic.h"
#include "Snac/ViscoPlastic/ViscoPlastic.h"
#include "Snac/Maxwell/Maxwell.h"
#include "Snac/Temperature/Temperature.h"
#include "SnacCuda.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define NO_HANDLE ((ExtensionInfo_Index)-1)

static int has_hook(void* context, Name ep, Name hook) {
    EntryPoint* e = Context_GetEntryPoint(context, ep);
    return e && Stg_ObjectList_Get(e->hooks, hook) != NULL;
}

int SnacCuda_Inspect(Snac_Context* context, SnacCuda_Context* self) {
    ExtensionManager* elementExt = context->mesh->elementExtensionMgr;
    int n = 0;

    /* the one constitutive plugin: its hook on Snac_EP_Constitutive is named by its Type */
    if (has_hook(context, Snac_EP_Constitutive, "SnacElastic")) {
        self->constitutive = SNAC_RHEOLOGY_ELASTIC;
        n++;
    }
    if (has_hook(context, Snac_EP_Constitutive, "SnacPlastic")) {
        self->constitutive = SNAC_RHEOLOGY_PLASTIC;
        n++;
    }
    if (has_hook(context, Snac_EP_Constitutive, "SnacViscoPlastic")) {
        self->constitutive = SNAC_RHEOLOGY_VISCOPLASTIC;
        n++;
    }
    if (has_hook(context, Snac_EP_Constitutive, "SnacMaxwell")) {
        self->constitutive = SNAC_RHEOLOGY_MAXWELL;
        n++;
    }
    if (n != 1) return SNAC_GPU_ENOTSUP;
    self->plasticElement = ExtensionManager_GetHandle(elementExt, "SnacPlastic");
    self->viscoPlasticElement = ExtensionManager_GetHandle(elementExt, "SnacViscoPlastic");
    self->maxwellElement = ExtensionManager_GetHandle(elementExt, "SnacMaxwell");
    self->temperatureNode = ExtensionManager_GetHandle(context->mesh->nodeExtensionMgr, "SnacTemperature");
    self->temperatureContext = ExtensionManager_GetHandle(context->extensionMgr, "SnacTemperature");
    self->temperature = self->temperatureNode != NO_HANDLE && self->temperatureContext != NO_HANDLE;
    if (self->constitutive == SNAC_RHEOLOGY_PLASTIC && self->plasticElement == NO_HANDLE) return SNAC_GPU_EINVAL;
    if (self->constitutive == SNAC_RHEOLOGY_VISCOPLASTIC && self->viscoPlasticElement == NO_HANDLE)
        return SNAC_GPU_EINVAL;
    if (self->constitutive == SNAC_RHEOLOGY_MAXWELL && self->maxwellElement == NO_HANDLE) return SNAC_GPU_EINVAL;
    self->ne = context->mesh->elementLocalCount;
    self->nn = context->mesh->nodeLocalCount;
    /* the visco-plastic hook's Drucker-Prager branch keeps a per-tet plastic strain tensor */
    self->druckerPrager = 0;
    if (self->constitutive == SNAC_RHEOLOGY_VISCOPLASTIC) {
        long long e;
        for (e = 0; e < self->ne && !self->druckerPrager; e++)
            if (context->materialProperty[Snac_Element_At(context, e)->material_I].yieldcriterion == druckerprager)
                self->druckerPrager = 1;
    }
    return 0;
}

static double* alloc_doubles(double** p, long long n) {
    if (!*p) *p = (double*)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
    return *p;
}

static SnacPlastic_Element* plastic_of(Snac_Context* context, SnacCuda_Context* self, Snac_Element* element) {
    return (SnacPlastic_Element*)ExtensionManager_Get(context->mesh->elementExtensionMgr, element, self->plasticElement);
}
static SnacViscoPlastic_Element* viscoplastic_of(Snac_Context* context, SnacCuda_Context* self, Snac_Element* element) {
    return (SnacViscoPlastic_Element*)ExtensionManager_Get(context->mesh->elementExtensionMgr, element,
                                                           self->viscoPlasticElement);
}
static SnacMaxwell_Element* maxwell_of(Snac_Context* context, SnacCuda_Context* self, Snac_Element* element) {
    return (SnacMaxwell_Element*)ExtensionManager_Get(context->mesh->elementExtensionMgr, element, self->maxwellElement);
}
static SnacTemperature_Node* temperature_of(Snac_Context* context, SnacCuda_Context* self, Snac_Node* node) {
    return (SnacTemperature_Node*)ExtensionManager_Get(context->mesh->nodeExtensionMgr, node, self->temperatureNode);
}

/* The conditions a CompositeVC applies, node by node, found by applying it
 * (VariableCondition_ApplyToIndex, the call UpdateNode.c:155-157 makes every
 * step) to each of its indices twice, from two different starting values: a
 * component it fixes ends with the same value both times.  Whatever the VC's
 * make-up (walls, all nodes, several VCs fixing one component), the result is
 * what the reference applies, last-VC-wins included. */
static void probe_velocity_bcs(Snac_Context* context, unsigned char* mask, double* value) {
    VariableCondition* vc = (VariableCondition*)context->velocityBCs;
    const double probeA[3] = {1.0e300, -2.0e299, 3.0e298}, probeB[3] = {-7.0e297, 5.0e296, -4.0e295};
    Index i;
    if (!vc) return;
    for (i = 0; i < vc->indexCount; i++) {
        Index n = vc->indexTbl[i];
        Snac_Node* node = Snac_Node_At(context, n);
        double keep[3], a[3], b[3];
        int d;
        memcpy(keep, node->velocity, sizeof keep);
        memcpy(node->velocity, probeA, sizeof probeA);
        VariableCondition_ApplyToIndex(vc, n, context);
        memcpy(a, node->velocity, sizeof a);
        memcpy(node->velocity, probeB, sizeof probeB);
        VariableCondition_ApplyToIndex(vc, n, context);
        memcpy(b, node->velocity, sizeof b);
        memcpy(node->velocity, keep, sizeof keep);
        for (d = 0; d < 3; d++)
            if (memcmp(&a[d], &b[d], sizeof(double)) == 0) {
                mask[n] |= (unsigned char)(1u << d);
                value[n * 3 + d] = a[d];
            }
    }
}

static void probe_temperature_bcs(Snac_Context* context, SnacCuda_Context* self, unsigned char* mask, double* value) {
    SnacTemperature_Context* tc =
        (SnacTemperature_Context*)ExtensionManager_Get(context->extensionMgr, context, self->temperatureContext);
    VariableCondition* vc = (VariableCondition*)tc->temperatureBCs;
    Index i;
    if (!vc) return;
    for (i = 0; i < vc->indexCount; i++) {
        Index n = vc->indexTbl[i];
        SnacTemperature_Node* t = temperature_of(context, self, Snac_Node_At(context, n));
        double keep = t->temperature, a, b;
        t->temperature = 1.0e300;
        VariableCondition_ApplyToIndex(vc, n, context);
        a = t->temperature;
        t->temperature = -7.0e297;
        VariableCondition_ApplyToIndex(vc, n, context);
        b = t->temperature;
        t->temperature = keep;
        if (memcmp(&a, &b, sizeof a) == 0) {
            mask[n] = 1;
            value[n] = a;
        }
    }
}

/* A scale c with RN(base[i] * c) == want[i] for every i (bit for bit), the
 * factor the device applies to a base phase's table; 1 when the tables are
 * equal.  Candidates: the quotient of the first non-zero pair and its
 * neighbours a few ulps away.  Returns 0 when there is none. */
static int find_scale(const double* base, const double* want, int n, double* scale) {
    int i, k, first = -1, same = 1;
    for (i = 0; i < n; i++) {
        if (memcmp(&base[i], &want[i], sizeof(double)) != 0) same = 0;
        if (first < 0 && base[i] != 0.0) first = i;
    }
    if (same) {
        *scale = 1.0;
        return 1;
    }
    if (first < 0) return 0;
    {
        double c = want[first] / base[first], lo = c, hi = c;
        for (k = 0; k < 9; k++) {
            const double cand = k == 0 ? c : (k % 2 ? (lo = nextafter(lo, -INFINITY)) : (hi = nextafter(hi, INFINITY)));
            int ok = 1;
            for (i = 0; i < n && ok; i++) {
                const double got = base[i] * cand;
                ok = memcmp(&got, &want[i], sizeof(double)) == 0;
            }
            if (ok) {
                *scale = cand;
                return 1;
            }
        }
    }
    return 0;
}

/* Everything but the cohesion and friction tables and the reference
 * viscosity: what phases sharing a base must have in common. */
static int same_shape(const snac_material* a, const snac_material* b, int dp_a, int dp_b, double tol_a, double tol_b) {
    snac_material x = *a, y = *b;
    memset(x.cohesion, 0, sizeof x.cohesion);
    memset(y.cohesion, 0, sizeof y.cohesion);
    memset(x.friction_angle, 0, sizeof x.friction_angle);
    memset(y.friction_angle, 0, sizeof y.friction_angle);
    x.refvisc = y.refvisc = 0.0;
    return memcmp(&x, &y, sizeof x) == 0 && dp_a == dp_b && memcmp(&tol_a, &tol_b, sizeof tol_a) == 0;
}

/* More phases than the device's table holds (SNAC_MAX_PHASES): the
 * reference expresses spatially varying strength or viscosity as one phase
 * per element (or per region).  Group the phases into base phases that
 * differ only by a factor on the cohesion table, the friction table and the
 * reference viscosity, and give every element its factors as per-element
 * scales, which the device applies to the base's values (the product
 * reproduces each phase's own value bit for bit, checked here).  A friction
 * scale makes the device evaluate sin and tan of the scaled angles itself
 * instead of taking the host's values. */
static int group_phases(snac_gpu_desc* d, SnacCuda_DescStore* st, long long ne) {
    const int nmat = d->n_materials;
    const int nseg1 = SNAC_MAX_SEGMENTS + 1;
    int* base_of = (int*)malloc(sizeof(int) * (size_t)nmat);
    double* cs = (double*)malloc(sizeof(double) * (size_t)nmat);
    double* fs = (double*)malloc(sizeof(double) * (size_t)nmat);
    double* vs = (double*)malloc(sizeof(double) * (size_t)nmat);
    int bases[SNAC_MAX_PHASES], nb = 0, p, b, need_c = 0, need_f = 0, need_v = 0, rc = 0;
    long long e;
    for (p = 0; p < nmat && !rc; p++) {
        const snac_material* m = &st->materials[p];
        base_of[p] = -1;
        for (b = 0; b < nb && base_of[p] < 0; b++) {
            const snac_material* r = &st->materials[bases[b]];
            if (!same_shape(m, r, st->dpMaxIterations[p], st->dpMaxIterations[bases[b]], st->dpTolerance[p],
                            st->dpTolerance[bases[b]]))
                continue;
            if (find_scale(r->cohesion, m->cohesion, nseg1, &cs[p]) &&
                find_scale(r->friction_angle, m->friction_angle, nseg1, &fs[p]) &&
                find_scale(&r->refvisc, &m->refvisc, 1, &vs[p]))
                base_of[p] = b;
        }
        if (base_of[p] < 0) {
            if (nb == SNAC_MAX_PHASES) {
                rc = SNAC_GPU_ENOTSUP; /* more distinct phases than scaled copies of 32 */
                break;
            }
            bases[nb] = p;
            base_of[p] = nb++;
            cs[p] = fs[p] = vs[p] = 1.0;
        }
        need_c |= cs[p] != 1.0;
        need_f |= fs[p] != 1.0;
        need_v |= vs[p] != 1.0;
    }
    if (!rc) {
        snac_material* mats = (snac_material*)calloc((size_t)nb, sizeof(snac_material));
        int* maxit = (int*)calloc((size_t)nb, sizeof(int));
        double* tol = (double*)calloc((size_t)nb, sizeof(double));
        for (b = 0; b < nb; b++) {
            mats[b] = st->materials[bases[b]];
            maxit[b] = st->dpMaxIterations[bases[b]];
            tol[b] = st->dpTolerance[bases[b]];
        }
        if (need_c) st->cohesionScale = (double*)malloc(sizeof(double) * (size_t)(ne > 0 ? ne : 1));
        if (need_f) st->frictionScale = (double*)malloc(sizeof(double) * (size_t)(ne > 0 ? ne : 1));
        if (need_v) st->viscScale = (double*)malloc(sizeof(double) * (size_t)(ne > 0 ? ne : 1));
        for (e = 0; e < ne; e++) {
            const int q = st->elementMaterial[e];
            if (need_c) st->cohesionScale[e] = cs[q];
            if (need_f) st->frictionScale[e] = fs[q];
            if (need_v) st->viscScale[e] = vs[q];
            st->elementMaterial[e] = base_of[q];
        }
        free(st->materials);
        free(st->dpMaxIterations);
        free(st->dpTolerance);
        st->materials = mats;
        st->dpMaxIterations = maxit;
        st->dpTolerance = tol;
        d->n_materials = nb;
        d->materials = mats;
        d->dp_max_iterations = maxit;
        d->dp_tolerance = tol;
        d->element_cohesion_scale = st->cohesionScale;
        d->element_friction_scale = st->frictionScale;
        d->element_visc_scale = st->viscScale;
    }
    free(base_of);
    free(cs);
    free(fs);
    free(vs);
    return rc;
}

void SnacCuda_FreeDescStore(SnacCuda_DescStore* st) {
    free(st->materials);
    free(st->elementMaterial);
    free(st->initStress);
    free(st->initVelocity);
    free(st->initTemperature);
    free(st->velocityBCMask);
    free(st->velocityBCValue);
    free(st->temperatureBCMask);
    free(st->temperatureBCValue);
    free(st->dpMaxIterations);
    free(st->dpTolerance);
    free(st->cohesionScale);
    free(st->frictionScale);
    free(st->viscScale);
    memset(st, 0, sizeof *st);
}

int SnacCuda_FillDesc(Snac_Context* context, SnacCuda_Context* self, snac_gpu_desc* d, SnacCuda_DescStore* st) {
    Mesh* mesh = context->mesh;
    HexaMD* decomp = (HexaMD*)context->meshLayout->decomp;
    BlockGeometry* geometry = (BlockGeometry*)context->meshLayout->elementLayout->geometry;
    const long long ne = self->ne, nn = self->nn;
    long long e, n;
    unsigned nmat = 0, p;
    int q, t;

    memset(d, 0, sizeof *d);
    memset(st, 0, sizeof *st);
    if (decomp->procsInUse != 1) return SNAC_GPU_ENOTSUP; /* the device model is the whole mesh */
    d->abi_version = SNAC_GPU_ABI_VERSION;
    d->nx = (int)decomp->elementGlobal3DCounts[0];
    d->ny = (int)decomp->elementGlobal3DCounts[1];
    d->nz = (int)decomp->elementGlobal3DCounts[2];
    if ((long long)d->nx * d->ny * d->nz != ne) return SNAC_GPU_EINVAL;
    for (q = 0; q < 3; q++) {
        d->min[q] = geometry->min[q];
        d->max[q] = geometry->max[q];
    }
    d->node_coords = (const double*)mesh->nodeCoord; /* Coord[nn]: x, y, z per node */

    d->dt_type = strcmp(context->dtType, Snac_DtType_Constant) == 0 ? SNAC_DT_CONSTANT
                 : strcmp(context->dtType, Snac_DtType_Wave) == 0   ? SNAC_DT_WAVE
                                                                    : SNAC_DT_DYNAMIC;
    d->dt = context->dt;
    d->strain_inert = context->strain_inert;
    d->gravity = context->gravity;
    d->demf = context->demf;
    d->constitutive = self->constitutive;
    d->temperature = self->temperature;
    d->compute_thermal_stress = context->computeThermalStress;
    d->hydrostatic_ic = 0;       /* the ICs ran on the host: their results are passed as initial values */
    d->temperature_sweep_ic = 0;
    d->pisos = context->pisos;
    d->rzbo = ne ? Snac_Element_At(context, 0)->rzbo : 0.0;
    d->winkler = has_hook(context, Snac_EP_Force, "SnacWinklerForce");
    d->traction_bc = has_hook(context, Snac_EP_Force, "SnacTractionBC");
    d->topo_kappa = context->topo_kappa;
    d->topo_grad_criterion = context->topoGradCriterion;

    /* phases: the materials the elements refer to */
    st->elementMaterial = (int*)malloc(sizeof(int) * (size_t)(ne > 0 ? ne : 1));
    for (e = 0; e < ne; e++) {
        st->elementMaterial[e] = (int)Snac_Element_At(context, e)->material_I;
        if (Snac_Element_At(context, e)->material_I + 1 > nmat) nmat = Snac_Element_At(context, e)->material_I + 1;
    }
    st->materials = (snac_material*)calloc(nmat ? nmat : 1, sizeof(snac_material));
    st->dpMaxIterations = (int*)calloc(nmat ? nmat : 1, sizeof(int));
    st->dpTolerance = (double*)calloc(nmat ? nmat : 1, sizeof(double));
    for (p = 0; p < nmat; p++) {
        const Snac_Material* m = &context->materialProperty[p];
        snac_material* o = &st->materials[p];
        unsigned s;
        o->density = m->phsDensity;
        o->alpha = m->alpha;
        o->beta = m->beta;
        o->lambda = m->lambda;
        o->mu = m->mu;
        o->yield_mohr_coulomb = m->yieldcriterion == mohrcoulomb;
        st->dpMaxIterations[p] = (int)m->maxiterations;
        st->dpTolerance[p] = m->constitutivetolerance;
        if (d->constitutive == SNAC_RHEOLOGY_PLASTIC || d->constitutive == SNAC_RHEOLOGY_VISCOPLASTIC) {
            if (m->nsegments > SNAC_MAX_SEGMENTS) return SNAC_GPU_ENOTSUP;
            o->nsegments = (int)m->nsegments;
            for (s = 0; s <= m->nsegments; s++) {
                o->plstrain[s] = m->plstrain[s];
                o->friction_angle[s] = m->frictionAngle[s];
                o->dilation_angle[s] = m->dilationAngle[s];
                o->cohesion[s] = m->cohesion[s];
            }
        }
        o->ten_off = m->ten_off;
        o->vis_min = m->vis_min;
        o->vis_max = m->vis_max;
        o->refvisc = m->refvisc;
        o->refsrate = m->refsrate;
        o->reftemp = m->reftemp;
        o->activation_e = m->activationE;
        o->srexponent = m->srexponent;
        o->thermal_conduct = m->thermal_conduct;
        o->heat_capacity = m->heatCapacity;
    }
    d->n_materials = (int)nmat;
    d->materials = st->materials;
    d->dp_max_iterations = st->dpMaxIterations;
    d->dp_tolerance = st->dpTolerance;
    d->element_material = st->elementMaterial;
    if (nmat > SNAC_MAX_PHASES) {
        int rc = group_phases(d, st, ne);
        if (rc) return rc;
    }

    /* the state after the ICs, as initial values */
    st->initStress = (double*)malloc(sizeof(double) * (size_t)(ne * Tetrahedra_Count * 6 + 1));
    for (e = 0; e < ne; e++) {
        Snac_Element* element = Snac_Element_At(context, e);
        for (t = 0; t < Tetrahedra_Count; t++) {
            double* o = &st->initStress[(e * Tetrahedra_Count + t) * 6];
            o[0] = element->tetra[t].stress[0][0];
            o[1] = element->tetra[t].stress[1][1];
            o[2] = element->tetra[t].stress[2][2];
            o[3] = element->tetra[t].stress[0][1];
            o[4] = element->tetra[t].stress[0][2];
            o[5] = element->tetra[t].stress[1][2];
        }
    }
    d->init_stress = st->initStress;
    st->initVelocity = (double*)malloc(sizeof(double) * (size_t)(nn * 3 + 1));
    for (n = 0; n < nn; n++)
        for (q = 0; q < 3; q++) st->initVelocity[n * 3 + q] = Snac_Node_At(context, n)->velocity[q];
    d->init_velocity = st->initVelocity;
    if (self->temperature) {
        /* temperature0 is the temperature before the BCs were applied
         * (temperature/VariableConditions.c:214-224); the device applies them again */
        st->initTemperature = (double*)malloc(sizeof(double) * (size_t)(nn + 1));
        for (n = 0; n < nn; n++) st->initTemperature[n] = temperature_of(context, self, Snac_Node_At(context, n))->temperature0;
        d->init_temperature = st->initTemperature;
    }

    /* boundary conditions, resolved per node */
    st->velocityBCMask = (unsigned char*)calloc((size_t)(nn + 1), 1);
    st->velocityBCValue = (double*)calloc((size_t)(nn * 3 + 1), sizeof(double));
    probe_velocity_bcs(context, st->velocityBCMask, st->velocityBCValue);
    d->node_velocity_bc_mask = st->velocityBCMask;
    d->node_velocity_bc_value = st->velocityBCValue;
    if (self->temperature) {
        st->temperatureBCMask = (unsigned char*)calloc((size_t)(nn + 1), 1);
        st->temperatureBCValue = (double*)calloc((size_t)(nn + 1), sizeof(double));
        probe_temperature_bcs(context, self, st->temperatureBCMask, st->temperatureBCValue);
        d->node_temperature_bc_mask = st->temperatureBCMask;
        d->node_temperature_bc_value = st->temperatureBCValue;
    }
    return 0;
}

void SnacCuda_Pack(Snac_Context* context, SnacCuda_Context* self) {
    const long long ne = self->ne, nn = self->nn;
    long long e, n;
    int q, t;
    alloc_doubles(&self->coord, nn * 3);
    alloc_doubles(&self->velocity, nn * 3);
    alloc_doubles(&self->stress, ne * Tetrahedra_Count * 6);
    alloc_doubles(&self->force, nn * 3);
    alloc_doubles(&self->inertialMass, nn);
    if (self->constitutive == SNAC_RHEOLOGY_PLASTIC || self->constitutive == SNAC_RHEOLOGY_VISCOPLASTIC)
        alloc_doubles(&self->plasticStrain, ne * Tetrahedra_Count);
    if (self->constitutive == SNAC_RHEOLOGY_VISCOPLASTIC || self->constitutive == SNAC_RHEOLOGY_MAXWELL)
        alloc_doubles(&self->viscosity, ne * Tetrahedra_Count);
    if (self->druckerPrager) alloc_doubles(&self->plasticStrainTensor, ne * Tetrahedra_Count * 6);
    if (self->temperature) alloc_doubles(&self->temperature_, nn);
    for (n = 0; n < nn; n++) {
        Snac_Node* node = Snac_Node_At(context, n);
        for (q = 0; q < 3; q++) {
            self->coord[n * 3 + q] = context->mesh->nodeCoord[n][q];
            self->velocity[n * 3 + q] = node->velocity[q];
        }
        if (self->temperature) self->temperature_[n] = temperature_of(context, self, node)->temperature;
    }
    for (e = 0; e < ne; e++) {
        Snac_Element* element = Snac_Element_At(context, e);
        for (t = 0; t < Tetrahedra_Count; t++) {
            double* o = &self->stress[(e * Tetrahedra_Count + t) * 6];
            o[0] = element->tetra[t].stress[0][0];
            o[1] = element->tetra[t].stress[1][1];
            o[2] = element->tetra[t].stress[2][2];
            o[3] = element->tetra[t].stress[0][1];
            o[4] = element->tetra[t].stress[0][2];
            o[5] = element->tetra[t].stress[1][2];
            if (self->constitutive == SNAC_RHEOLOGY_PLASTIC)
                self->plasticStrain[e * Tetrahedra_Count + t] = plastic_of(context, self, element)->plasticStrain[t];
            if (self->constitutive == SNAC_RHEOLOGY_VISCOPLASTIC) {
                SnacViscoPlastic_Element* vp = viscoplastic_of(context, self, element);
                self->plasticStrain[e * Tetrahedra_Count + t] = vp->plasticStrain[t];
                self->viscosity[e * Tetrahedra_Count + t] = vp->viscosity[t];
            }
            if (self->druckerPrager) {
                SnacViscoPlastic_Element* vp = viscoplastic_of(context, self, element);
                double* q = &self->plasticStrainTensor[(e * Tetrahedra_Count + t) * 6];
                q[0] = vp->plasticstrainTensor[t][0][0];
                q[1] = vp->plasticstrainTensor[t][1][1];
                q[2] = vp->plasticstrainTensor[t][2][2];
                q[3] = vp->plasticstrainTensor[t][0][1];
                q[4] = vp->plasticstrainTensor[t][0][2];
                q[5] = vp->plasticstrainTensor[t][1][2];
            }
            if (self->constitutive == SNAC_RHEOLOGY_MAXWELL)
                self->viscosity[e * Tetrahedra_Count + t] = maxwell_of(context, self, element)->viscosity[t];
        }
    }
}

void SnacCuda_Unpack(Snac_Context* context, SnacCuda_Context* self) {
    const long long ne = self->ne, nn = self->nn;
    long long e, n;
    int q, t;
    for (n = 0; n < nn; n++) {
        Snac_Node* node = Snac_Node_At(context, n);
        for (q = 0; q < 3; q++) {
            context->mesh->nodeCoord[n][q] = self->coord[n * 3 + q];
            node->velocity[q] = self->velocity[n * 3 + q];
            node->force[q] = self->force[n * 3 + q];
        }
        node->inertialMass = self->inertialMass[n];
        if (self->temperature) temperature_of(context, self, node)->temperature = self->temperature_[n];
    }
    for (e = 0; e < ne; e++) {
        Snac_Element* element = Snac_Element_At(context, e);
        for (t = 0; t < Tetrahedra_Count; t++) {
            const double* o = &self->stress[(e * Tetrahedra_Count + t) * 6];
            element->tetra[t].stress[0][0] = o[0];
            element->tetra[t].stress[1][1] = o[1];
            element->tetra[t].stress[2][2] = o[2];
            element->tetra[t].stress[0][1] = o[3];
            element->tetra[t].stress[0][2] = o[4];
            element->tetra[t].stress[1][2] = o[5];
            if (self->constitutive == SNAC_RHEOLOGY_PLASTIC)
                plastic_of(context, self, element)->plasticStrain[t] = self->plasticStrain[e * Tetrahedra_Count + t];
            if (self->constitutive == SNAC_RHEOLOGY_VISCOPLASTIC) {
                SnacViscoPlastic_Element* vp = viscoplastic_of(context, self, element);
                vp->plasticStrain[t] = self->plasticStrain[e * Tetrahedra_Count + t];
                vp->viscosity[t] = self->viscosity[e * Tetrahedra_Count + t];
            }
            if (self->druckerPrager) {
                SnacViscoPlastic_Element* vp = viscoplastic_of(context, self, element);
                const double* q = &self->plasticStrainTensor[(e * Tetrahedra_Count + t) * 6];
                vp->plasticstrainTensor[t][0][0] = q[0];
                vp->plasticstrainTensor[t][1][1] = q[1];
                vp->plasticstrainTensor[t][2][2] = q[2];
                vp->plasticstrainTensor[t][0][1] = q[3];
                vp->plasticstrainTensor[t][0][2] = q[4];
                vp->plasticstrainTensor[t][1][2] = q[5];
            }
            if (self->constitutive == SNAC_RHEOLOGY_MAXWELL)
                maxwell_of(context, self, element)->viscosity[t] = self->viscosity[e * Tetrahedra_Count + t];
        }
    }
}
