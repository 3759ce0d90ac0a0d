/*
 * ref_driver.c — drives the reference's OWN hot-path functions, compiled from
 * the SNAC source tree against oracle/refshim (see oracle/Makefile), through
 * the same interface as the restated oracle (snac_oracle.h, with the prefix
 * "ref_" instead of "so_").
 *
 * TEST INFRASTRUCTURE ONLY.  What is restated here is the glue the reference
 * keeps in StGermain / Context.c, which cannot be built without MPI and
 * libxml2: mesh tables (HexaEL.c:456-573), the loop drivers
 * (Context.c:978-1036, 1063-1184), Sync (Context.c:1208-1268) and the plugin
 * ICs.  Every per-element / per-node computation is the reference's code:
 * Snac_UpdateElementMomentum, Snac_StrainRate, Snac_Stress,
 * Snac_Force, Snac_UpdateNodeMomentum_PreProcess, Snac_UpdateNodeMomentum,
 * the topography hooks, the four constitutive hooks, the temperature loops
 * and _SnacHydroStaticIC_IC.
 */
#define _GNU_SOURCE
#include <stdarg.h>
#include <dlfcn.h>
#ifdef REF_THREADS
#include <pthread.h>
#endif

#include "common/snac_shim_core.h"
#include "common/snac_shim_plastic.h"
#include "common/snac_shim_viscoplastic.h"
#include "common/snac_shim_maxwell.h"
#include "common/snac_shim_temperature.h"
#include "common/snac_shim_hydro.h"
#include "common/snac_shim_winkler.h"
#include "common/snac_shim_traction.h"
#include "../include/snac_gpu.h"

/* winkler/Register.c's globals (used by its spherical variant only) */
double Spherical_RMin, Spherical_RMax;

void SnacPlastic_Constitutive(void* context, Element_LocalIndex element_lI);
void SnacViscoPlastic_Constitutive(void* context, Element_LocalIndex element_lI);
void _SnacMaxwell_Constitutive(void* context, Element_LocalIndex element_lI);
void _SnacElastic_Constitutive(void* context, Element_LocalIndex element_lI);

/* names the reference compares by pointer (Context.c:70-82) */
const Name Snac_DtType_Constant = "constant";
const Name Snac_DtType_Dynamic = "dynamic";
const Name Snac_DtType_Wave = "wave";
const Name Snac_EP_LoopElementsEnergy = "Snac_EP_LoopElementsEnergy";
const Name Snac_EP_LoopNodesEnergy = "Snac_EP_LoopNodesEnergy";
const Name Snac_EP_CalcStresses = "Snac_EP_CalcStresses";
const Name Snac_EP_Constitutive = "Snac_EP_Constitutive";
const Name Snac_EP_LoopNodesMomentum = "Snac_EP_LoopNodesMomentum";
const Name Snac_EP_Force = "Snac_EP_Force";
const Name Snac_EP_LoopElementsMomentum = "Snac_EP_LoopElementsMomentum";
/* AbstractContext.c:58-69 */
const Name AbstractContext_EP_Initialise = "Context_Initialise";
const Name AbstractContext_EP_Dt = "Context_Dt";
const Name AbstractContext_EP_Solve = "Context_Solve";
const Name AbstractContext_EP_Sync = "Context_Sync";
const Name AbstractContext_EP_Dump = "Context_Dump";
const Type Snac_Context_Type = "Snac_Context";

/* ---- entry points (EntryPoint.c:681-850 semantics on a fixed-size list) ---------- */
void* Stg_ObjectList_Get(void* list, Name name) {
    Stg_ObjectList* l = (Stg_ObjectList*)list;
    for (unsigned i = 0; l && i < l->count; i++)
        if (strcmp(l->data[i]->name, name) == 0) return l->data[i];
    return NULL;
}
static Hook* hook_new(Stg_ObjectList* l, Name name, Func_Ptr f, Hook_AddedBy by) {
    for (int k = 0; k < SHIM_MAX_HOOKS; k++) {
        int used = 0;
        for (unsigned i = 0; i < l->count; i++) used |= l->data[i] == &l->store[k];
        if (!used) {
            l->store[k] = (Hook){name, f, by};
            return &l->store[k];
        }
    }
    shim_firewall("entry point: more than %d hooks", SHIM_MAX_HOOKS);
    return NULL;
}
static void list_insert(Stg_ObjectList* l, unsigned at, Hook* h) {
    if (!h) return;
    for (unsigned i = l->count; i > at; i--) l->data[i] = l->data[i - 1];
    l->data[at] = h;
    l->count++;
}
static int list_find(Stg_ObjectList* l, Name name) {
    for (unsigned i = 0; i < l->count; i++)
        if (strcmp(l->data[i]->name, name) == 0) return (int)i;
    return -1;
}
void EntryPoint_Append(void* ep, Name name, Func_Ptr f, Hook_AddedBy by) {
    EntryPoint* e = (EntryPoint*)ep;
    list_insert(e->hooks, e->hooks->count, hook_new(e->hooks, name, f, by));
}
void EntryPoint_Prepend(void* ep, Name name, Func_Ptr f, Hook_AddedBy by) {
    EntryPoint* e = (EntryPoint*)ep;
    list_insert(e->hooks, 0, hook_new(e->hooks, name, f, by));
}
void EntryPoint_InsertBefore(void* ep, Name before, Name name, Func_Ptr f, Hook_AddedBy by) {
    EntryPoint* e = (EntryPoint*)ep;
    int i = list_find(e->hooks, before);
    if (i < 0) {
        shim_firewall("EntryPoint_InsertBefore: no hook \"%s\" on %s", before, e->name);
        return;
    }
    list_insert(e->hooks, (unsigned)i, hook_new(e->hooks, name, f, by));
}
void EntryPoint_Replace(void* ep, Name old, Name name, Func_Ptr f, Hook_AddedBy by) {
    EntryPoint* e = (EntryPoint*)ep;
    int i = list_find(e->hooks, old);
    if (i < 0) {
        shim_firewall("EntryPoint_Replace: no hook \"%s\" on %s", old, e->name);
        return;
    }
    e->hooks->data[i]->name = name;
    e->hooks->data[i]->funcPtr = f;
    e->hooks->data[i]->addedBy = by;
}
void EntryPoint_ReplaceAll(void* ep, Name name, Func_Ptr f, Hook_AddedBy by) {
    EntryPoint* e = (EntryPoint*)ep;
    e->hooks->count = 0;
    EntryPoint_Append(ep, name, f, by);
}
void EntryPoint_Remove(void* ep, Name name) {
    EntryPoint* e = (EntryPoint*)ep;
    int i = list_find(e->hooks, name);
    if (i < 0) return;
    for (unsigned k = (unsigned)i; k + 1 < e->hooks->count; k++) e->hooks->data[k] = e->hooks->data[k + 1];
    e->hooks->count--;
}
EntryPoint* shim_get_entry_point(void* context, Name name) {
    Snac_Context* c = (Snac_Context*)context;
    for (unsigned i = 0; i < c->shim_ep_count; i++)
        if (strcmp(c->shim_eps[i].name, name) == 0) return &c->shim_eps[i];
    return NULL;
}

/* ---- extension managers ------------------------------------------------------------ */
ExtensionInfo_Index ExtensionManager_GetHandle(void* mgr, Name name) {
    ExtensionManager* m = (ExtensionManager*)mgr;
    for (unsigned k = 0; k < SHIM_MAX_EXTENSIONS; k++)
        if (m->name[k] && strcmp(m->name[k], name) == 0) return k;
    return (ExtensionInfo_Index)-1;
}
ExtensionInfo_Index ExtensionManager_Add(void* mgr, Name name, size_t size) {
    ExtensionManager* m = (ExtensionManager*)mgr;
    for (unsigned k = 0; k < SHIM_MAX_EXTENSIONS; k++)
        if (!m->ext[k]) {
            m->ext[k] = calloc(m->count ? m->count : 1, size ? size : 1);
            m->extsize[k] = size;
            m->name[k] = name;
            m->owned |= 1u << k;
            return k;
        }
    shim_firewall("ExtensionManager_Add: no free slot for %s", name);
    return (ExtensionInfo_Index)-1;
}

ExtensionInfo_Index SnacPlastic_ElementHandle = 0;
ExtensionInfo_Index SnacViscoPlastic_ElementHandle = 1;
ExtensionInfo_Index SnacMaxwell_ElementHandle = 2;
ExtensionInfo_Index SnacTemperature_ElementHandle = 3;
ExtensionInfo_Index SnacTemperature_NodeHandle = 0;
ExtensionInfo_Index SnacTemperature_ContextHandle = 0;

/* printf of the visco-plastic hook (compiled with -Dprintf=shim_quiet_printf):
 * its messages are dropped, nothing it computes depends on them */
int shim_quiet_printf(const char* restrict fmt, ...) {
    (void)fmt;
    return 0;
}

int shim_firewall_count = 0;
char shim_firewall_msg[512];
void shim_firewall(const char* fmt, ...) {
    if (shim_firewall_count++ == 0) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(shim_firewall_msg, sizeof shim_firewall_msg, fmt, ap);
        va_end(ap);
    }
}

typedef struct ref_ctx {
    Snac_Context ctx;
    Mesh mesh;
    MeshLayout layout;
    HexaMD decomp;
    ElementLayout elayout;
    BlockGeometry geom;
    Dictionary dict;
    ExtensionManager emgr, nmgr, cmgr;
    Stream stream;
    SnacTemperature_Context tctx;
    VariableCondition vbc, tbc;
    unsigned char* vbc_mask;
    double (*vbc_val)[3];
    unsigned char* tbc_mask;
    double* tbc_val;
    int nx, ny, nz, nnx, nny, nnz, constitutive, temperature, nmat;
    unsigned ne, nn;
    void (*hook)(void*, Element_LocalIndex);
    SnacPlastic_Element* pl;
    SnacViscoPlastic_Element* vp;
    SnacMaxwell_Element* mx;
    SnacTemperature_Element* te;
    SnacTemperature_Node* tn;
    double vmax;
    double currentTime; /* AbstractContext.c:871, 891 */
    int winkler, traction;
    double (*mass_store);
    double (*balance_store)[3];
    long timeStep_total;
    int verbatim_bc; /* VariableCondition_ApplyToIndex searches its index table as the reference does */
} ref_ctx;

static ref_ctx* g_current; /* the constitutive trampoline needs the hook */

/* Threads of the element and node loops.  Built with REF_THREADS
 * (_ref/libsnacref_mt.so) the loops whose iterations are independent in the
 * reference (every element or node writes only its own record; the minimum
 * length scale is a min, which does not round) run on this many threads,
 * each on one contiguous range, and give the serial build's bits; built
 * without it the loops are the serial ones. */
static int g_threads = 1;
void ref_set_threads(int n) { g_threads = n < 1 ? 1 : (n > 256 ? 256 : n); }
void ref_set_verbatim_bc(ref_ctx* r, int on) { r->verbatim_bc = on != 0; }
int ref_threads(void) {
#ifdef REF_THREADS
    return g_threads;
#else
    return 1;
#endif
}

typedef void (*range_fn)(ref_ctx* r, unsigned lo, unsigned hi, double* acc);
typedef struct { range_fn fn; ref_ctx* r; unsigned lo, hi; double acc; } range_job;
#ifdef REF_THREADS
static void* range_main(void* p) {
    range_job* j = (range_job*)p;
    j->fn(j->r, j->lo, j->hi, &j->acc);
    return NULL;
}
#endif
/* fn over [lo, hi) split into contiguous ranges, one per thread (a range
 * whose thread could not be started runs on the caller); returns the min of
 * the ranges' accumulators, each started at acc0 */
static double parallel_range(range_fn fn, ref_ctx* r, unsigned lo, unsigned hi, int threads, double acc0) {
    double acc = acc0;
#ifdef REF_THREADS
    if (threads > 1 && hi - lo >= (unsigned)threads) {
        range_job job[256];
        pthread_t tid[256];
        int started[256];
        const unsigned long long n = hi - lo;
        for (int t = 0; t < threads; t++) {
            job[t] = (range_job){fn, r, lo + (unsigned)(n * t / threads), lo + (unsigned)(n * (t + 1) / threads), acc0};
            started[t] = t > 0 && pthread_create(&tid[t], NULL, range_main, &job[t]) == 0;
        }
        fn(r, job[0].lo, job[0].hi, &job[0].acc);
        for (int t = 1; t < threads; t++) {
            if (started[t])
                pthread_join(tid[t], NULL);
            else
                fn(r, job[t].lo, job[t].hi, &job[t].acc);
        }
        for (int t = 0; t < threads; t++)
            if (job[t].acc < acc) acc = job[t].acc;
        return acc;
    }
#else
    (void)threads;
#endif
    fn(r, lo, hi, &acc);
    return acc;
}

static void run_constitutive(void* ep, void* ctx, Element_LocalIndex e) {
    (void)ep;
    g_current->hook(ctx, e);
}

/* VariableCondition_ApplyToIndex (StGermain VariableCondition.c:449-463)
 * first finds the index in the condition's index table by a linear search
 * and returns when it is absent; the table of a CompositeVC is the union of
 * its walls' node sets in ascending node order.  The per-node masks below
 * give the same result in O(1); with verbatim_bc the search runs first, as
 * in the reference, so that its cost can be timed. */
static int vc_has_index(const VariableCondition* vc, Index n) {
    Index q;
    for (q = 0; q < vc->indexCount; q++)
        if (vc->indexTbl[q] == n) break;
    return q < vc->indexCount;
}
static void vbc_apply_index(VariableCondition* vc, Index n, void* context) {
    ref_ctx* r = (ref_ctx*)((char*)vc - offsetof(ref_ctx, vbc));
    (void)context;
    if (r->verbatim_bc && !vc_has_index(vc, n)) return;
    for (int d = 0; d < 3; d++)
        if (r->vbc_mask[n] & (1u << d)) r->mesh.node[n].velocity[d] = r->vbc_val[n][d];
}
static void vbc_apply(VariableCondition* vc, void* context) {
    for (Index q = 0; q < vc->indexCount; q++) vbc_apply_index(vc, vc->indexTbl[q], context);
}
static void tbc_apply_index(VariableCondition* vc, Index n, void* context) {
    ref_ctx* r = (ref_ctx*)((char*)vc - offsetof(ref_ctx, tbc));
    (void)context;
    if (r->verbatim_bc && !vc_has_index(vc, n)) return;
    if (r->tbc_mask[n]) r->tn[n].temperature = r->tbc_val[n];
}
static void tbc_apply(VariableCondition* vc, void* context) {
    for (Index q = 0; q < vc->indexCount; q++) tbc_apply_index(vc, vc->indexTbl[q], context);
}
static Element_GlobalIndex id_map(void* decomp, Element_LocalIndex lI) {
    (void)decomp;
    return lI;
}

static int wall_has(const ref_ctx* r, int wall, int i, int j, int k) {
    switch (wall) {
        case SNAC_WALL_BACK: return k == 0;
        case SNAC_WALL_LEFT: return i == 0;
        case SNAC_WALL_BOTTOM: return j == 0;
        case SNAC_WALL_RIGHT: return i == r->nnx - 1;
        case SNAC_WALL_TOP: return j == r->nny - 1;
        case SNAC_WALL_FRONT: return k == r->nnz - 1;
        case SNAC_WALL_ALL: return 1;
        default: return 0;
    }
}

void ref_destroy(ref_ctx* r);
int ref_time_step_zero(ref_ctx* r);
int ref_loop_elements_energy(ref_ctx* r);
int ref_loop_nodes_energy(ref_ctx* r);
int ref_calc_stresses(ref_ctx* r);
int ref_loop_nodes_momentum(ref_ctx* r);
int ref_loop_elements_momentum(ref_ctx* r);
int ref_sync(ref_ctx* r);

/* ---- the context's named entry points with the reference's default hooks -------------
 * (Context.c:470-600, the plugins' Register.c).  The checker's own step
 * (ref_step) calls the loops directly; these serve the plugin host below,
 * which drives a context the way AbstractContext does, through whatever
 * hooks the entry points hold. */
enum { EP_INIT, EP_DT, EP_SOLVE, EP_SYNC, EP_DUMP, EP_LEE, EP_LNE, EP_CALC, EP_CONST, EP_LNM, EP_FORCE, EP_LEM, EP_N };
typedef void (*void_hook)(void*);
static void run_hooks(void* c, Name ep) {
    EntryPoint* e = Context_GetEntryPoint(c, ep);
    for (unsigned i = 0; e && i < e->hooks->count && !shim_firewall_count; i++) ((void_hook)e->hooks->data[i]->funcPtr)(c);
}
static void hk_time_step_zero(void* c, void* data) { (void)data; ref_time_step_zero((ref_ctx*)c); }
static double hk_dt(void* c) { return ((Snac_Context*)c)->dt; } /* _Snac_Context_Dt */
static void hk_loop_elements_energy(void* c) { ref_loop_elements_energy((ref_ctx*)c); }
static void hk_loop_nodes_energy(void* c) { ref_loop_nodes_energy((ref_ctx*)c); }
static void hk_calc_stresses(void* c) { ref_calc_stresses((ref_ctx*)c); }
static void hk_loop_nodes_momentum(void* c) { ref_loop_nodes_momentum((ref_ctx*)c); }
static void hk_loop_elements_momentum(void* c) { ref_loop_elements_momentum((ref_ctx*)c); }
static void hk_sync(void* c) { ref_sync((ref_ctx*)c); }
/* _Snac_Context_Solve, Context.c:1063-1099 (one rank: no Mesh_Sync) */
static void hk_solve(void* c) {
    run_hooks(c, Snac_EP_LoopElementsEnergy);
    run_hooks(c, Snac_EP_LoopNodesEnergy);
    run_hooks(c, Snac_EP_CalcStresses);
    run_hooks(c, Snac_EP_LoopNodesMomentum);
    run_hooks(c, Snac_EP_LoopElementsMomentum);
}
static void no_hook(void* c) { (void)c; }

static void setup_entry_points(ref_ctx* r, Name constitutive_type) {
    static const char* names[EP_N];
    names[EP_INIT] = AbstractContext_EP_Initialise;
    names[EP_DT] = AbstractContext_EP_Dt;
    names[EP_SOLVE] = AbstractContext_EP_Solve;
    names[EP_SYNC] = AbstractContext_EP_Sync;
    names[EP_DUMP] = AbstractContext_EP_Dump;
    names[EP_LEE] = Snac_EP_LoopElementsEnergy;
    names[EP_LNE] = Snac_EP_LoopNodesEnergy;
    names[EP_CALC] = Snac_EP_CalcStresses;
    names[EP_CONST] = Snac_EP_Constitutive;
    names[EP_LNM] = Snac_EP_LoopNodesMomentum;
    names[EP_FORCE] = Snac_EP_Force;
    names[EP_LEM] = Snac_EP_LoopElementsMomentum;
    Snac_Context* c = &r->ctx;
    c->shim_eps = calloc(EP_N, sizeof(EntryPoint));
    c->shim_ep_count = EP_N;
    for (int i = 0; i < EP_N; i++) {
        c->shim_eps[i].name = names[i];
        c->shim_eps[i].hooks = &c->shim_eps[i].list;
    }
    EntryPoint* e = c->shim_eps;
    EntryPoint_Append(&e[EP_INIT], "SnacTimeStepZero", (Func_Ptr)hk_time_step_zero, "Snac");
    EntryPoint_Append(&e[EP_DT], "SnacDt", (Func_Ptr)hk_dt, "Snac");
    EntryPoint_Append(&e[EP_SOLVE], "SnacSolve", (Func_Ptr)hk_solve, "Snac");
    EntryPoint_Append(&e[EP_SYNC], "SnacSync", (Func_Ptr)hk_sync, "Snac");
    if (r->temperature) {
        EntryPoint_Append(&e[EP_LEE], "SnacTemperature", (Func_Ptr)hk_loop_elements_energy, "SnacTemperature");
        EntryPoint_Append(&e[EP_LNE], "SnacTemperature", (Func_Ptr)hk_loop_nodes_energy, "SnacTemperature");
    }
    EntryPoint_Append(&e[EP_CALC], "default", (Func_Ptr)hk_calc_stresses, "Snac");
    EntryPoint_Append(&e[EP_CONST], constitutive_type, (Func_Ptr)no_hook, constitutive_type);
    EntryPoint_Append(&e[EP_LNM], "default", (Func_Ptr)hk_loop_nodes_momentum, "Snac");
    EntryPoint_Append(&e[EP_FORCE], "default", (Func_Ptr)no_hook, "Snac");
    if (r->winkler) EntryPoint_Append(&e[EP_FORCE], "SnacWinklerForce", (Func_Ptr)no_hook, "SnacWinklerForce");
    if (r->traction) EntryPoint_Append(&e[EP_FORCE], "SnacTractionBC", (Func_Ptr)no_hook, "SnacTractionBC");
    EntryPoint_Append(&e[EP_LEM], "default", (Func_Ptr)hk_loop_elements_momentum, "Snac");
}

ref_ctx* ref_create(const snac_gpu_desc* d, int* status) {
    *status = SNAC_GPU_EINVAL;
    if (!d || d->nx < 1 || d->ny < 1 || d->nz < 1 || d->n_materials < 1) return NULL;
    ref_ctx* r = (ref_ctx*)calloc(1, sizeof *r);
    Snac_Context* c = &r->ctx;
    shim_firewall_count = 0;
    r->nx = d->nx;
    r->ny = d->ny;
    r->nz = d->nz;
    r->nnx = d->nx + 1;
    r->nny = d->ny + 1;
    r->nnz = d->nz + 1;
    r->ne = (unsigned)(d->nx * d->ny * d->nz);
    r->nn = (unsigned)(r->nnx * r->nny * r->nnz);
    r->constitutive = d->constitutive;
    r->temperature = d->temperature;
    /* mesh */
    Mesh* m = &r->mesh;
    m->layout = &r->layout;
    r->layout.decomp = &r->decomp;
    r->layout.elementLayout = &r->elayout;
    r->elayout.geometry = &r->geom;
    for (int q = 0; q < 3; q++) {
        r->geom.min[q] = d->min[q];
        r->geom.max[q] = d->max[q];
    }
    r->decomp.nodeGlobal3DCounts[0] = r->nnx;
    r->decomp.nodeGlobal3DCounts[1] = r->nny;
    r->decomp.nodeGlobal3DCounts[2] = r->nnz;
    r->decomp.elementGlobal3DCounts[0] = r->nx;
    r->decomp.elementGlobal3DCounts[1] = r->ny;
    r->decomp.elementGlobal3DCounts[2] = r->nz;
    r->decomp.partition3DCounts[0] = r->decomp.partition3DCounts[1] = r->decomp.partition3DCounts[2] = 1;
    r->decomp.elementLocal3DCounts[0][0] = r->nx;
    r->decomp.elementLocal3DCounts[0][1] = r->ny;
    r->decomp.elementLocal3DCounts[0][2] = r->nz;
    r->decomp.procsInUse = 1;
    r->decomp.elementMapLocalToGlobal = id_map;
    m->nodeLocalCount = m->nodeDomainCount = r->nn;
    m->elementLocalCount = m->elementDomainCount = r->ne;
    m->node = calloc(r->nn, sizeof(Snac_Node));
    m->element = calloc(r->ne, sizeof(Snac_Element));
    m->nodeCoord = calloc(r->nn, sizeof(Coord));
    m->nodeL2G = calloc(r->nn, sizeof(Node_GlobalIndex));
    m->elementNodeTbl = calloc(r->ne, sizeof(Node_DomainIndex*));
    m->nodeElementTbl = calloc(r->nn, sizeof(Element_DomainIndex*));
    m->nodeElementCountTbl = calloc(r->nn, sizeof(Node_ElementIndex));
    m->nodeNeighbourTbl = calloc(r->nn, sizeof(Node_DomainIndex*));
    r->vbc_mask = calloc(r->nn, 1);
    r->vbc_val = calloc(r->nn, sizeof *r->vbc_val);
    r->tbc_mask = calloc(r->nn, 1);
    r->tbc_val = calloc(r->nn, sizeof(double));
    r->vbc.indexTbl = calloc(r->nn, sizeof(Index));
    r->tbc.indexTbl = calloc(r->nn, sizeof(Index));
    r->mass_store = calloc(r->nn, sizeof(double));
    r->balance_store = calloc(r->nn, sizeof(double[3]));
    for (unsigned e = 0; e < r->ne; e++) {
        unsigned i = e % r->nx, j = (e / r->nx) % r->ny, k = e / (r->nx * r->ny);
        static const int off[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                                      {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
        m->elementNodeTbl[e] = calloc(8, sizeof(Node_DomainIndex));
        for (int q = 0; q < 8; q++)
            m->elementNodeTbl[e][q] = (i + off[q][0]) + (j + off[q][1]) * r->nnx + (k + off[q][2]) * r->nnx * r->nny;
    }
    for (unsigned n = 0; n < r->nn; n++) {
        int i = n % r->nnx, j = (n / r->nnx) % r->nny, k = n / (r->nnx * r->nny);
        m->nodeL2G[n] = n;
        m->nodeElementCountTbl[n] = 8;
        m->nodeElementTbl[n] = calloc(8, sizeof(Element_DomainIndex));
        for (int q = 0; q < 8; q++) {
            int dx = q & 1, dy = (q >> 1) & 1, dz = (q >> 2) & 1;
            int ei = i - 1 + dx, ej = j - 1 + dy, ek = k - 1 + dz;
            if (ei < 0 || ej < 0 || ek < 0 || ei >= r->nx || ej >= r->ny || ek >= r->nz)
                m->nodeElementTbl[n][q] = r->ne; /* elementCount, skipped by the hooks */
            else
                m->nodeElementTbl[n][q] = ei + ej * r->nx + ek * r->nx * r->ny;
        }
        m->nodeNeighbourTbl[n] = calloc(6, sizeof(Node_DomainIndex));
        /* IJK6Topology.c:283-345: +x, +y, +z, -x, -y, -z; off the mesh = invalid (>= node count) */
        {
            const int step[6][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {-1, 0, 0}, {0, -1, 0}, {0, 0, -1}};
            for (int q = 0; q < 6; q++) {
                int a = i + step[q][0], b = j + step[q][1], cz = k + step[q][2];
                m->nodeNeighbourTbl[n][q] = (a < 0 || b < 0 || cz < 0 || a >= r->nnx || b >= r->nny || cz >= r->nnz)
                                                ? (Node_DomainIndex)r->nn
                                                : (Node_DomainIndex)(a + b * r->nnx + cz * r->nnx * r->nny);
            }
        }
        /* coordinates: BlockGeometry.c:326-349 */
        int ijk[3] = {i, j, k}, size[3] = {r->nnx, r->nny, r->nnz};
        for (int q = 0; q < 3; q++) {
            if (d->node_coords)
                m->nodeCoord[n][q] = d->node_coords[n * 3 + q];
            else
                m->nodeCoord[n][q] = size[q] > 1 ? d->min[q] + (d->max[q] - d->min[q]) * ((double)ijk[q] / (double)(size[q] - 1))
                                                 : d->min[q];
        }
        for (int b = 0; b < d->n_velocity_bcs; b++) {
            const snac_wall_bc* bc = &d->velocity_bcs[b];
            if (!wall_has(r, bc->wall, i, j, k)) continue;
            for (int q = 0; q < 3; q++)
                if (bc->mask & (1 << q)) {
                    r->vbc_mask[n] |= (unsigned char)(1u << q);
                    r->vbc_val[n][q] = bc->value[q];
                }
        }
        if (r->vbc_mask[n]) r->vbc.indexTbl[r->vbc.indexCount++] = n;
        for (int b = 0; b < d->n_temperature_bcs; b++) {
            const snac_wall_bc* bc = &d->temperature_bcs[b];
            if (!wall_has(r, bc->wall, i, j, k) || !(bc->mask & 1)) continue;
            r->tbc_mask[n] = 1;
            r->tbc_val[n] = bc->value[0];
        }
        if (r->tbc_mask[n]) r->tbc.indexTbl[r->tbc.indexCount++] = n;
        if (d->init_velocity)
            for (int q = 0; q < 3; q++) m->node[n].velocity[q] = d->init_velocity[n * 3 + q];
    }
    r->vbc.applyToIndex = vbc_apply_index;
    r->vbc.apply = vbc_apply;
    r->tbc.applyToIndex = tbc_apply_index;
    r->tbc.apply = tbc_apply;
    /* extensions */
    r->pl = calloc(r->ne, sizeof *r->pl);
    r->vp = calloc(r->ne, sizeof *r->vp);
    r->mx = calloc(r->ne, sizeof *r->mx);
    r->te = calloc(r->ne, sizeof *r->te);
    r->tn = calloc(r->nn, sizeof *r->tn);
    r->emgr.base = (char*)m->element;
    r->emgr.stride = sizeof(Snac_Element);
    r->emgr.ext[0] = (char*)r->pl;
    r->emgr.extsize[0] = sizeof *r->pl;
    r->emgr.ext[1] = (char*)r->vp;
    r->emgr.extsize[1] = sizeof *r->vp;
    r->emgr.ext[2] = (char*)r->mx;
    r->emgr.extsize[2] = sizeof *r->mx;
    r->emgr.ext[3] = (char*)r->te;
    r->emgr.extsize[3] = sizeof *r->te;
    r->nmgr.base = (char*)m->node;
    r->nmgr.stride = sizeof(Snac_Node);
    r->nmgr.ext[0] = (char*)r->tn;
    r->nmgr.extsize[0] = sizeof *r->tn;
    r->cmgr.base = (char*)c;
    r->cmgr.stride = 1;
    r->cmgr.ext[0] = (char*)&r->tctx;
    r->cmgr.extsize[0] = sizeof r->tctx;
    r->emgr.count = r->ne;
    r->nmgr.count = r->nn;
    r->cmgr.count = 1;
    /* the loaded plugins' extension keys (their Type names) */
    if (d->constitutive == SNAC_RHEOLOGY_PLASTIC) r->emgr.name[0] = "SnacPlastic";
    if (d->constitutive == SNAC_RHEOLOGY_VISCOPLASTIC) r->emgr.name[1] = "SnacViscoPlastic";
    if (d->constitutive == SNAC_RHEOLOGY_MAXWELL) r->emgr.name[2] = "SnacMaxwell";
    if (d->temperature) r->emgr.name[3] = r->nmgr.name[0] = r->cmgr.name[0] = "SnacTemperature";
    m->elementExtensionMgr = &r->emgr;
    m->nodeExtensionMgr = &r->nmgr;
    /* context */
    c->mesh = m;
    c->meshLayout = &r->layout;
    c->dictionary = &r->dict;
    c->outputPath = ".";
    c->extensionMgr = &r->cmgr;
    c->snacError = c->snacInfo = c->debug = c->info = c->verbose = &r->stream;
    c->forceCalcType = Snac_Force_Complete;
    c->dtType = d->dt_type == SNAC_DT_CONSTANT ? Snac_DtType_Constant
                : d->dt_type == SNAC_DT_WAVE   ? Snac_DtType_Wave
                                               : Snac_DtType_Dynamic;
    c->dt = d->dt;
    c->strain_inert = d->strain_inert;
    c->gravity = d->gravity;
    r->winkler = d->winkler;
    r->traction = d->traction_bc;
    c->demf = d->demf;
    c->topo_kappa = d->topo_kappa;
    c->topoGradCriterion = d->topo_grad_criterion;
    c->computeThermalStress = d->compute_thermal_stress;
    c->velocityBCs = &r->vbc;
    c->constitutiveK = 0;
    c->shim_ep_run[0] = (void*)run_constitutive;
    r->tctx.topTemp = d->top_temp;
    r->tctx.bottomTemp = d->bottom_temp;
    r->tctx.temperatureBCs = &r->tbc;
    Name ctype = "SnacElastic";
    switch (d->constitutive) {
        case SNAC_RHEOLOGY_ELASTIC: r->hook = _SnacElastic_Constitutive; break;
        case SNAC_RHEOLOGY_PLASTIC: r->hook = SnacPlastic_Constitutive; ctype = "SnacPlastic"; break;
        case SNAC_RHEOLOGY_VISCOPLASTIC: r->hook = SnacViscoPlastic_Constitutive; ctype = "SnacViscoPlastic"; break;
        case SNAC_RHEOLOGY_MAXWELL: r->hook = _SnacMaxwell_Constitutive; ctype = "SnacMaxwell"; break;
        default: ref_destroy(r); return NULL;
    }
    setup_entry_points(r, ctype);
    /* materials (Context.c:826-914), per-element multipliers as one phase per element */
    int per_elem = d->element_cohesion_scale || d->element_friction_scale || d->element_visc_scale;
    if (per_elem && d->constitutive == SNAC_RHEOLOGY_MAXWELL) {
        *status = SNAC_GPU_ENOTSUP;
        ref_destroy(r);
        return NULL;
    }
    int nmat = per_elem ? (int)r->ne : d->n_materials;
    c->materialProperty = calloc(nmat, sizeof(Snac_Material));
    r->nmat = nmat;
    for (int p = 0; p < nmat; p++) {
        int src = per_elem ? (d->element_material ? d->element_material[p] : 0) : p;
        if (src < 0 || src >= d->n_materials) {
            *status = SNAC_GPU_EMATERIAL;
            ref_destroy(r);
            return NULL;
        }
        const snac_material* sm = &d->materials[src];
        Snac_Material* mm = &c->materialProperty[p];
        mm->rheology = Snac_Material_Elastic;
        mm->phsDensity = sm->density;
        mm->alpha = sm->alpha;
        mm->beta = sm->beta;
        mm->lambda = sm->lambda;
        mm->mu = sm->mu;
        mm->yieldcriterion = sm->yield_mohr_coulomb ? mohrcoulomb : druckerprager;
        mm->maxiterations = d->dp_max_iterations ? (unsigned)d->dp_max_iterations[src] : 1u; /* Context.c:851-854 */
        mm->constitutivetolerance = d->dp_tolerance ? d->dp_tolerance[src] : 1.e-3;
        mm->nsegments = sm->nsegments;
        mm->plstrain = calloc(sm->nsegments + 1, sizeof(double));
        mm->frictionAngle = calloc(sm->nsegments + 1, sizeof(double));
        mm->dilationAngle = calloc(sm->nsegments + 1, sizeof(double));
        mm->cohesion = calloc(sm->nsegments + 1, sizeof(double));
        for (int i = 0; i <= sm->nsegments; i++) {
            mm->plstrain[i] = sm->plstrain[i];
            mm->frictionAngle[i] = sm->friction_angle[i];
            mm->dilationAngle[i] = sm->dilation_angle[i];
            mm->cohesion[i] = sm->cohesion[i];
            if (per_elem && d->element_cohesion_scale) mm->cohesion[i] = mm->cohesion[i] * d->element_cohesion_scale[p];
            if (per_elem && d->element_friction_scale)
                mm->frictionAngle[i] = mm->frictionAngle[i] * d->element_friction_scale[p];
        }
        mm->ten_off = sm->ten_off;
        mm->vis_min = sm->vis_min;
        mm->vis_max = sm->vis_max;
        mm->refvisc = sm->refvisc;
        if (per_elem && d->element_visc_scale) mm->refvisc = mm->refvisc * d->element_visc_scale[p];
        mm->refsrate = sm->refsrate;
        mm->reftemp = sm->reftemp;
        mm->activationE = sm->activation_e;
        mm->srexponent = sm->srexponent;
        mm->thermal_conduct = sm->thermal_conduct;
        mm->heatCapacity = sm->heat_capacity;
    }
    /* elementICs: phase and stress */
    for (unsigned e = 0; e < r->ne; e++) {
        Snac_Element* el = &m->element[e];
        el->material_I = per_elem ? e : (unsigned)(d->element_material ? d->element_material[e] : 0);
        if (d->init_stress)
            for (int t = 0; t < Tetrahedra_Count; t++) {
                const double* q = &d->init_stress[(e * Tetrahedra_Count + t) * 6];
                el->tetra[t].stress[0][0] = q[0];
                el->tetra[t].stress[1][1] = q[1];
                el->tetra[t].stress[2][2] = q[2];
                el->tetra[t].stress[0][1] = q[3];
                el->tetra[t].stress[0][2] = q[4];
                el->tetra[t].stress[1][2] = q[5];
            }
    }
    g_current = r;
    /* nodeICs: temperature */
    if (d->temperature)
        for (unsigned n = 0; n < r->nn; n++) {
            if (d->temperature_sweep_ic)
                _SnacTemperature_Top2BottomSweep(n, 0, c, &r->tn[n].temperature);
            else if (d->init_temperature)
                r->tn[n].temperature = d->init_temperature[n];
        }
    /* VariableCondition_Apply(velocityBCs), Context.c:773 */
    vbc_apply(&r->vbc, c);
    /* plugin ICs before SnacTimeStepZero, in load order */
    if (d->temperature) _SnacTemperature_InitialConditions(c);
    if (d->constitutive == SNAC_RHEOLOGY_PLASTIC) {
        for (int p = 0; p < nmat; p++) c->materialProperty[p].rheology |= Snac_Material_Plastic;
        /* plasticStrain = 0 (calloc) */
    }
    if (d->constitutive == SNAC_RHEOLOGY_VISCOPLASTIC) {
        double dtm = 0;
        for (int p = 0; p < nmat; p++) {
            c->materialProperty[p].rheology |= Snac_Material_ViscoPlastic;
            double v = 9.0e-01 * c->materialProperty[p].vis_min / c->materialProperty[p].mu;
            dtm = (p == 0) ? v : (v < dtm ? v : dtm);
        }
        if (c->dt > dtm && c->dtType != Snac_DtType_Constant) c->dt = dtm;
        for (unsigned e = 0; e < r->ne; e++)
            for (int t = 0; t < Tetrahedra_Count; t++)
                r->vp[e].viscosity[t] = c->materialProperty[m->element[e].material_I].vis_min;
    }
    if (d->constitutive == SNAC_RHEOLOGY_MAXWELL) {
        c->materialProperty[0].rheology |= Snac_Material_Maxwell;
        double dtm = 1.0e-01 * c->materialProperty[0].vis_min / c->materialProperty[0].mu;
        if (c->dt > dtm && c->dtType != Snac_DtType_Constant) c->dt = dtm;
    }
    if (d->hydrostatic_ic) _SnacHydroStaticIC_IC(c);
    c->timeStep = 0;
    *status = shim_firewall_count ? SNAC_GPU_EPHYSICS : 0;
    return r;
}

void ref_destroy(ref_ctx* r) {
    if (!r) return;
    Mesh* m = &r->mesh;
    for (unsigned e = 0; e < r->ne && m->elementNodeTbl; e++) free(m->elementNodeTbl[e]);
    for (unsigned n = 0; n < r->nn && m->nodeElementTbl; n++) {
        free(m->nodeElementTbl[n]);
        free(m->nodeNeighbourTbl[n]);
    }
    for (int p = 0; p < r->nmat && r->ctx.materialProperty; p++) {
        free(r->ctx.materialProperty[p].plstrain);
        free(r->ctx.materialProperty[p].frictionAngle);
        free(r->ctx.materialProperty[p].dilationAngle);
        free(r->ctx.materialProperty[p].cohesion);
    }
    free(r->ctx.materialProperty);
    free(m->node);
    free(m->element);
    free(m->nodeCoord);
    free(m->nodeL2G);
    free(m->elementNodeTbl);
    free(m->nodeElementTbl);
    free(m->nodeElementCountTbl);
    free(m->nodeNeighbourTbl);
    free(r->vbc_mask);
    free(r->vbc_val);
    free(r->tbc_mask);
    free(r->tbc_val);
    free(r->vbc.indexTbl);
    free(r->tbc.indexTbl);
    free(r->pl);
    free(r->vp);
    free(r->mx);
    free(r->te);
    free(r->tn);
    free(r->mass_store);
    free(r->balance_store);
    ExtensionManager* mgrs[3] = {&r->emgr, &r->nmgr, &r->cmgr};
    for (int q = 0; q < 3; q++)
        for (unsigned k = 0; k < SHIM_MAX_EXTENSIONS; k++)
            if (mgrs[q]->owned & (1u << k)) free(mgrs[q]->ext[k]);
    free(r->ctx.shim_eps);
    free(r);
}

static int status_of(void) { return shim_firewall_count ? SNAC_GPU_ENAN : 0; }

/* _Snac_Context_LoopElements, Context.c:1156-1184 */
static void elements_momentum_range(ref_ctx* r, unsigned lo, unsigned hi, double* mn) {
    for (unsigned e = lo; e < hi; e++) {
        double ls;
        Snac_UpdateElementMomentum(&r->ctx, e, &ls);
        if (ls < *mn) *mn = ls;
    }
}
int ref_loop_elements_momentum(ref_ctx* r) {
    Snac_Context* c = &r->ctx;
    g_current = r;
    Snac_UpdateElementMomentum(c, 0, &c->minLengthScale);
    c->minLengthScale = parallel_range(elements_momentum_range, r, 1, r->ne, g_threads, c->minLengthScale);
    return status_of();
}

/* _Snac_Context_CalcStresses, Context.c:1102-1117 */
static void calc_stresses_range(ref_ctx* r, unsigned lo, unsigned hi, double* unused) {
    (void)unused;
    for (unsigned e = lo; e < hi; e++) {
        Snac_StrainRate(&r->ctx, e);
        Snac_Stress(&r->ctx, e);
    }
}
int ref_calc_stresses(ref_ctx* r) {
    g_current = r;
    parallel_range(calc_stresses_range, r, 0, r->ne, g_threads, 0.0);
    return status_of();
}

/* _Snac_Context_LoopNodes, Context.c:1120-1154, with the hook order of Context.c:568-593 */
static void node_forces_range(ref_ctx* r, unsigned lo, unsigned hi, double* unused) {
    Snac_Context* c = &r->ctx;
    (void)unused;
    for (unsigned n = lo; n < hi; n++) {
        Snac_Node* node = &r->mesh.node[n];
        Snac_Force(c, n, c->speedOfSound, &r->mass_store[n], &node->inertialMass, &node->force, &r->balance_store[n]);
        if (r->winkler)  /* appended to Snac_EP_Force, winkler/Register.c:140-145 */
            _SnacWinklerForce_Apply(c, n, c->speedOfSound, &r->mass_store[n], &node->inertialMass, &node->force,
                                    &r->balance_store[n]);
        if (r->traction)  /* tractionBC/Register.c:79-83 */
            _SnacTractionBC_Force_Apply(c, n, c->speedOfSound, &r->mass_store[n], &node->inertialMass, &node->force,
                                        &r->balance_store[n]);
    }
}
static void node_update_range(ref_ctx* r, unsigned lo, unsigned hi, double* unused) {
    Snac_Context* c = &r->ctx;
    (void)unused;
    for (unsigned n = lo; n < hi; n++) {
        Snac_Node* node = &r->mesh.node[n];
        Snac_UpdateNodeMomentum_PreProcess(c, n, node->inertialMass, node->force);
        Snac_UpdateNodeMomentum(c, n, node->inertialMass, node->force);
        Snac_UpdateNodeMomentum_DiffTopo(c, n, node->inertialMass, node->force);
        Snac_UpdateNodeMomentum_UpdateInteriorTopo(c, n, node->inertialMass, node->force);
        Snac_UpdateNodeMomentum_AdjustEdgeTopo(c, n, node->inertialMass, node->force);
    }
}
int ref_loop_nodes_momentum(ref_ctx* r) {
    Snac_Context* c = &r->ctx;
    g_current = r;
    parallel_range(node_forces_range, r, 0, r->nn, g_threads, 0.0);
    /* the topography hooks walk the top surface in node order (UpdateNode.c:161-857):
     * the update loop stays serial unless they are certain to do nothing */
    const int topo_idle = c->topo_kappa == 0 && c->topoGradMax < c->topoGradCriterion;
    parallel_range(node_update_range, r, 0, r->nn, topo_idle ? g_threads : 1, 0.0);
    return status_of();
}

int ref_loop_elements_energy(ref_ctx* r) {
    g_current = r;
    if (r->temperature) SnacTemperature_LoopElements(&r->ctx);
    return status_of();
}

int ref_loop_nodes_energy(ref_ctx* r) {
    g_current = r;
    if (r->temperature) SnacTemperature_LoopNodes(&r->ctx);
    return status_of();
}

/* _Snac_Context_Sync, Context.c:1208-1268 (one rank) */
int ref_sync(ref_ctx* r) {
    Snac_Context* c = &r->ctx;
    double v, vx, vy, vz, vmax = 0.0f, vlb = 3.0e-11f;
    for (Index q = 0; q < r->vbc.indexCount; q++) {
        Snac_Node* node = &r->mesh.node[r->vbc.indexTbl[q]];
        vx = node->velocity[0];
        vy = node->velocity[1];
        vz = node->velocity[2];
        v = sqrt(vx * vx + vy * vy + vz * vz);
        if (v > vmax) vmax = v;
    }
    if (vmax < vlb) vmax = vlb;
    r->vmax = vmax;
    if (c->timeStep == 0 && c->restartTimestep == 0) c->initMinLengthScale = c->minLengthScale;
    if (c->dtType == Snac_DtType_Dynamic) {
        c->dt = c->minLengthScale * 0.45f * c->strain_inert / vmax;
        c->speedOfSound = c->minLengthScale * 0.5f / c->dt;
    } else if (c->dtType == Snac_DtType_Wave) {
        c->dt = 0.5f * c->minLengthScale / c->speedOfSound;
    }
    return status_of();
}

/* Snac_Context_TimeStepZero, Context.c:978-1036 */
int ref_time_step_zero(ref_ctx* r) {
    g_current = r;
    for (unsigned e = 0; e < r->ne; e++) {
        Snac_Element* el = &r->mesh.element[e];
        double phsDensity = r->ctx.materialProperty[el->material_I].phsDensity, sVolAvg = 0.0f;
        el->stress = 0;
        for (int t = 0; t < Tetrahedra_Count; t++) {
            sVolAvg += el->tetra[t].stress[1][1] * el->tetra[t].stress[2][2] +
                       el->tetra[t].stress[2][2] * el->tetra[t].stress[0][0] +
                       el->tetra[t].stress[0][0] * el->tetra[t].stress[1][1];
            el->tetra[t].avgTemp = 0.0f;
            el->tetra[t].density = phsDensity;
        }
        el->stress = 0.5f * sqrt(0.5f * fabs(sVolAvg / Tetrahedra_Count));
    }
    ref_loop_elements_momentum(r);
    return ref_sync(r);
}

int ref_begin_step(ref_ctx* r) {
    r->ctx.timeStep++;
    r->ctx.dt = 1.0 * r->ctx.dt;
    r->currentTime += r->ctx.dt;
    return status_of();
}

int ref_step(ref_ctx* r, int nsteps) {
    for (int i = 0; i < nsteps && !shim_firewall_count; i++) {
        ref_begin_step(r);
        ref_loop_elements_energy(r);
        ref_loop_nodes_energy(r);
        ref_calc_stresses(r);
        ref_loop_nodes_momentum(r);
        ref_loop_elements_momentum(r);
        ref_sync(r);
    }
    return status_of();
}

/* ---- state access, same layout as snac_state_view ---------------------------------- */
int ref_get_state(ref_ctx* r, const snac_state_view* v) {
    for (unsigned n = 0; n < r->nn; n++) {
        for (int q = 0; q < 3; q++) {
            if (v->coord) v->coord[n * 3 + q] = r->mesh.nodeCoord[n][q];
            if (v->velocity) v->velocity[n * 3 + q] = r->mesh.node[n].velocity[q];
            if (v->force) v->force[n * 3 + q] = r->mesh.node[n].force[q];
        }
        if (v->temperature) v->temperature[n] = r->tn[n].temperature;
        if (v->inertial_mass) v->inertial_mass[n] = r->mesh.node[n].inertialMass;
    }
    for (unsigned e = 0; e < r->ne; e++)
        for (int t = 0; t < Tetrahedra_Count; t++) {
            const Snac_Element_Tetrahedra* tt = &r->mesh.element[e].tetra[t];
            if (v->stress) {
                double* q = &v->stress[((size_t)e * Tetrahedra_Count + t) * 6];
                q[0] = tt->stress[0][0];
                q[1] = tt->stress[1][1];
                q[2] = tt->stress[2][2];
                q[3] = tt->stress[0][1];
                q[4] = tt->stress[0][2];
                q[5] = tt->stress[1][2];
            }
            double ps = 0, vis = 0;
            if (r->constitutive == SNAC_RHEOLOGY_PLASTIC) ps = r->pl[e].plasticStrain[t];
            if (r->constitutive == SNAC_RHEOLOGY_VISCOPLASTIC) {
                ps = r->vp[e].plasticStrain[t];
                vis = r->vp[e].viscosity[t];
            }
            if (r->constitutive == SNAC_RHEOLOGY_MAXWELL) vis = r->mx[e].viscosity[t];
            if (v->plastic_strain) v->plastic_strain[e * Tetrahedra_Count + t] = ps;
            if (v->viscosity) v->viscosity[e * Tetrahedra_Count + t] = vis;
            if (v->plastic_strain_tensor) {
                double* q = &v->plastic_strain_tensor[((size_t)e * Tetrahedra_Count + t) * 6];
                const StrainTensor* p = &r->vp[e].plasticstrainTensor[t];
                q[0] = (*p)[0][0];
                q[1] = (*p)[1][1];
                q[2] = (*p)[2][2];
                q[3] = (*p)[0][1];
                q[4] = (*p)[0][2];
                q[5] = (*p)[1][2];
            }
        }
    return 0;
}

int ref_set_state(ref_ctx* r, const snac_state_view* v) {
    for (unsigned n = 0; n < r->nn; n++) {
        for (int q = 0; q < 3; q++) {
            if (v->coord) r->mesh.nodeCoord[n][q] = v->coord[n * 3 + q];
            if (v->velocity) r->mesh.node[n].velocity[q] = v->velocity[n * 3 + q];
        }
        if (v->temperature) r->tn[n].temperature = v->temperature[n];
    }
    for (unsigned e = 0; e < r->ne; e++)
        for (int t = 0; t < Tetrahedra_Count; t++) {
            Snac_Element_Tetrahedra* tt = &r->mesh.element[e].tetra[t];
            if (v->stress) {
                const double* q = &v->stress[((size_t)e * Tetrahedra_Count + t) * 6];
                tt->stress[0][0] = q[0];
                tt->stress[1][1] = q[1];
                tt->stress[2][2] = q[2];
                tt->stress[0][1] = q[3];
                tt->stress[0][2] = q[4];
                tt->stress[1][2] = q[5];
            }
            if (v->plastic_strain) {
                r->pl[e].plasticStrain[t] = v->plastic_strain[e * Tetrahedra_Count + t];
                r->vp[e].plasticStrain[t] = v->plastic_strain[e * Tetrahedra_Count + t];
            }
            if (v->plastic_strain_tensor) {
                const double* q = &v->plastic_strain_tensor[((size_t)e * Tetrahedra_Count + t) * 6];
                StrainTensor* p = &r->vp[e].plasticstrainTensor[t];
                (*p)[0][0] = q[0];
                (*p)[1][1] = q[1];
                (*p)[2][2] = q[2];
                (*p)[0][1] = q[3];
                (*p)[0][2] = q[4];
                (*p)[1][2] = q[5];
            }
        }
    return 0;
}

void ref_scalars(ref_ctx* r, snac_scalars* o) {
    o->dt = r->ctx.dt;
    o->min_length_scale = r->ctx.minLengthScale;
    o->vmax = r->vmax;
    o->speed_of_sound = r->ctx.speedOfSound;
    o->time_step = r->ctx.timeStep;
    o->current_time = r->currentTime;
}

void ref_set_dt(ref_ctx* r, double dt) { r->ctx.dt = dt; }

const char* ref_last_error(ref_ctx* r) {
    (void)r;
    return shim_firewall_count ? shim_firewall_msg : "";
}

void ref_get_geometry(ref_ctx* r, double* volume, double* area, double* normal) {
    for (unsigned e = 0; e < r->ne; e++)
        for (int t = 0; t < Tetrahedra_Count; t++) {
            const Snac_Element_Tetrahedra* tt = &r->mesh.element[e].tetra[t];
            size_t et = (size_t)e * Tetrahedra_Count + t;
            if (volume) volume[et] = tt->volume;
            for (int f = 0; f < 4; f++) {
                if (area) area[et * 4 + f] = tt->surface[f].area;
                if (normal)
                    for (int q = 0; q < 3; q++) normal[(et * 4 + f) * 3 + q] = tt->surface[f].normal[q];
            }
        }
}

void ref_get_element_scalars(ref_ctx* r, double* volume, double* strain_rate, double* stress, double* hydro_pressure,
                             double* aps, double* min_length_scale) {
    for (unsigned e = 0; e < r->ne; e++) {
        const Snac_Element* el = &r->mesh.element[e];
        if (volume) volume[e] = el->volume;
        if (strain_rate) strain_rate[e] = el->strainRate;
        if (stress) stress[e] = el->stress;
        if (hydro_pressure) hydro_pressure[e] = el->hydroPressure;
        if (aps)
            aps[e] = r->constitutive == SNAC_RHEOLOGY_PLASTIC        ? r->pl[e].aps
                     : r->constitutive == SNAC_RHEOLOGY_VISCOPLASTIC ? r->vp[e].aps
                                                                     : 0.0;
        if (min_length_scale) min_length_scale[e] = 0.0; /* not kept per element by the reference */
    }
}

void ref_get_tet_fields(ref_ctx* r, double* strain_rate, double* strain, double* density, double* avg_temp) {
    static const int ia[6] = {0, 1, 2, 0, 0, 1}, ib[6] = {0, 1, 2, 1, 2, 2};
    for (unsigned e = 0; e < r->ne; e++)
        for (int t = 0; t < Tetrahedra_Count; t++) {
            const Snac_Element_Tetrahedra* tt = &r->mesh.element[e].tetra[t];
            size_t et = (size_t)e * Tetrahedra_Count + t;
            for (int c6 = 0; c6 < 6; c6++) {
                if (strain_rate) strain_rate[et * 6 + c6] = tt->strainRate[ia[c6]][ib[c6]];
                if (strain) strain[et * 6 + c6] = tt->strain[ia[c6]][ib[c6]];
            }
            if (density) density[et] = tt->density;
            if (avg_temp) avg_temp[et] = tt->avgTemp;
        }
}

void ref_get_node_fields(ref_ctx* r, double* mass, double* balance) {
    for (unsigned n = 0; n < r->nn; n++) {
        if (mass) mass[n] = r->mass_store[n];
        if (balance)
            for (int q = 0; q < 3; q++) balance[n * 3 + q] = r->balance_store[n][q];
    }
}

/* ---- plugin host: a context driven through its entry points ---------------------------
 * What StGermain's PluginLoader and AbstractContext do for one rank
 * (PluginLoader.c:359-370, AbstractContext.c:874-941): find the plugin's
 * register function by name, let it submit its component, construct it
 * against this context, then run Initialise, the steps and Dump through the
 * hooks the entry points hold. */
typedef struct PluginEntry { Name type; void* (*defaultNew)(Name); } PluginEntry;
static PluginEntry g_submitted[8];
static int g_n_submitted;
Index PluginsManager_Submit(void* pm, Name codeletName, Name version, void* (*defaultNew)(Name)) {
    (void)pm;
    (void)version;
    if (g_n_submitted >= 8) return (Index)-1;
    g_submitted[g_n_submitted] = (PluginEntry){codeletName, defaultNew};
    return (Index)g_n_submitted++;
}
void* _Codelet_New(SizeT size, Type type, void* del, void* print, void* copy, void* defaultNew, void* construct,
                   void* build, void* init, void* execute, void* destroy, Name name) {
    (void)del, (void)print, (void)copy, (void)defaultNew, (void)build, (void)init, (void)execute, (void)destroy;
    Codelet* c = calloc(1, size > sizeof(Codelet) ? size : sizeof(Codelet));
    c->type = type;
    c->name = name;
    c->_construct = (Stg_Component_ConstructFunction*)construct;
    return c;
}
static Stg_Component* factory_construct_by_name(void* cf, Name name, Type type, Bool essential, void* data) {
    (void)type, (void)essential, (void)data;
    return strcmp(name, "context") == 0 ? (Stg_Component*)((Stg_ComponentFactory*)cf)->context : NULL;
}

/* loads plugin "name" (e.g. "SnacCuda") into the context: returns 0 or a negative status */
int ref_host_load_plugin(ref_ctx* r, const char* name) {
    char sym[128];
    Dl_info info;
    void* self = NULL;
    if (dladdr((void*)ref_create, &info) && info.dli_fname) self = dlopen(info.dli_fname, RTLD_NOW | RTLD_NOLOAD);
    if (!self) return SNAC_GPU_EINVAL;
    snprintf(sym, sizeof sym, "%s_Register", name);
    Index (*reg)(void*) = (Index(*)(void*))dlsym(self, sym);
    if (!reg) {  /* leading-underscore fallback, PluginLoader.c:365-370 */
        snprintf(sym, sizeof sym, "_%s_Register", name);
        reg = (Index(*)(void*))dlsym(self, sym);
    }
    dlclose(self);
    if (!reg) return SNAC_GPU_ENOTSUP;
    int before = g_n_submitted;
    reg(NULL);
    if (g_n_submitted != before + 1) return SNAC_GPU_EINVAL;
    Codelet* comp = (Codelet*)g_submitted[before].defaultNew((Name)name);
    g_n_submitted = before;
    Stg_ComponentFactory cf = {&r->ctx, factory_construct_by_name};
    comp->_construct(comp, &cf, NULL);
    free(comp);
    return shim_firewall_count ? SNAC_GPU_EPHYSICS : 0;
}

/* AbstractContext_Initialise: the Initialise hooks (SnacTimeStepZero, or its replacement) */
int ref_host_initialise(ref_ctx* r) {
    EntryPoint* e = Context_GetEntryPoint(&r->ctx, AbstractContext_EP_Initialise);
    for (unsigned i = 0; i < e->hooks->count && !shim_firewall_count; i++)
        ((void (*)(void*, void*))e->hooks->data[i]->funcPtr)(&r->ctx, NULL);
    return status_of();
}

/* nsteps x (timeStep++, dt from the Dt hook, currentTime += dt, Solve hooks, Sync hooks) */
int ref_host_step(ref_ctx* r, int nsteps) {
    Snac_Context* c = &r->ctx;
    for (int i = 0; i < nsteps && !shim_firewall_count; i++) {
        c->timeStep++;
        EntryPoint* dt = Context_GetEntryPoint(c, AbstractContext_EP_Dt);
        double d = c->dt;
        for (unsigned k = 0; k < dt->hooks->count; k++) d = ((double (*)(void*))dt->hooks->data[k]->funcPtr)(c);
        r->currentTime += d;
        c->dt = d; /* _setDt */
        run_hooks(c, AbstractContext_EP_Solve);
        run_hooks(c, AbstractContext_EP_Sync);
    }
    return status_of();
}

/* AbstractContext_Dump: the Dump hooks */
int ref_host_dump(ref_ctx* r) {
    run_hooks(&r->ctx, AbstractContext_EP_Dump);
    return status_of();
}

/* the hook names of one entry point, comma-separated (for tests) */
int ref_host_hooks(ref_ctx* r, const char* ep, char* out, int cap) {
    EntryPoint* e = Context_GetEntryPoint(&r->ctx, ep);
    if (!e || cap < 1) return SNAC_GPU_EINVAL;
    out[0] = 0;
    for (unsigned i = 0; i < e->hooks->count; i++) {
        if (i) strncat(out, ",", (size_t)cap - strlen(out) - 1);
        strncat(out, e->hooks->data[i]->name, (size_t)cap - strlen(out) - 1);
    }
    return 0;
}

/* the context, and a context extension by key (for the plugin's tests) */
void* ref_host_context(ref_ctx* r) { return &r->ctx; }
void* ref_host_extension(ref_ctx* r, const char* name) {
    ExtensionInfo_Index k = ExtensionManager_GetHandle(&r->cmgr, name);
    return k == (ExtensionInfo_Index)-1 ? NULL : r->cmgr.ext[k];
}
