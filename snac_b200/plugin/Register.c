/*
 * Register.c — the SnacCuda plugin's registration and its entry-point hooks.
 *
 * Registration follows the pattern of every SNAC plugin
 * (Snac/plugins/plastic/Register.c:49-98): _SnacCuda_Register submits the
 * component's default constructor to the PluginsManager; _SnacCuda_Construct
 * retrieves the context, adds the plugin's context extension and swaps the
 * hot loop's hooks for calls into libsnac_b200 (EntryPoint_Replace,
 * StGermain/Base/Extensibility/src/EntryPoint.c:735).  Every hook turns a
 * failing status into Journal_Firewall on context->snacError, as the
 * reference's own checks do.
 */
#include <mpi.h>
#include <StGermain/StGermain.h>
#include <StGermain/FD/FD.h>
#include "Snac/Snac.h"
#include "SnacCuda.h"
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

const Type SnacCuda_Type = "SnacCuda";
ExtensionInfo_Index SnacCuda_ContextHandle;

Index _SnacCuda_Register(PluginsManager* pluginsMgr) {
    return PluginsManager_Submit(pluginsMgr, SnacCuda_Type, "0", _SnacCuda_DefaultNew);
}

void* _SnacCuda_DefaultNew(Name name) {
    return _Codelet_New(sizeof(Codelet), SnacCuda_Type, _Codelet_Delete, _Codelet_Print, _Codelet_Copy,
                        _SnacCuda_DefaultNew, _SnacCuda_Construct, _Codelet_Build, _Codelet_Initialise,
                        _Codelet_Execute, _Codelet_Destroy, name);
}

static SnacCuda_Context* cuda_of(void* context) {
    Snac_Context* self = (Snac_Context*)context;
    return (SnacCuda_Context*)ExtensionManager_Get(self->extensionMgr, self, SnacCuda_ContextHandle);
}

/* a non-zero status from the library ends the run like the reference's firewalls */
static void cuda_check(Snac_Context* context, SnacCuda_Context* self, int rc, const char* what) {
    Journal_Firewall(rc == 0, context->snacError, "SnacCuda: %s returned %d: %s (element/node %lld)\n", what, rc,
                     self->gpu ? snac_gpu_last_error(self->gpu) : "no device model",
                     self->gpu ? snac_gpu_error_index(self->gpu) : -1LL);
}

/* The scalars the host loop reads back after each Sync: the next dt
 * (_Snac_Context_Dt returns context->dt), the minimum length scale and the
 * speed of sound. */
static void scalars_to_context(Snac_Context* context, SnacCuda_Context* self) {
    snac_scalars s;
    cuda_check(context, self, snac_gpu_scalars(self->gpu, &s), "snac_gpu_scalars");
    context->dt = s.dt;
    context->minLengthScale = s.min_length_scale;
    context->speedOfSound = s.speed_of_sound;
}

/* Replaces "SnacTimeStepZero" (Context.c:978-1036): the plugin ICs have run
 * on the host; the device model is built from that state and step zero runs
 * there. */
void SnacCuda_TimeStepZero(void* _context, void* data) {
    Snac_Context* context = (Snac_Context*)_context;
    SnacCuda_Context* self = cuda_of(context);
    snac_gpu_desc desc;
    SnacCuda_DescStore store;
    int rc;
    (void)data;

    rc = SnacCuda_Inspect(context, self);
    cuda_check(context, self, rc, "SnacCuda_Inspect");
    if (rc) return;
    rc = SnacCuda_FillDesc(context, self, &desc, &store);
    if (rc == 0) rc = snac_gpu_create(&desc, &self->gpu);
    SnacCuda_FreeDescStore(&store);
    cuda_check(context, self, rc, "snac_gpu_create");
    if (rc) return;
    /* plastic strain and viscosity as the plugin ICs left them (a restart may carry non-zero values) */
    SnacCuda_Pack(context, self);
    {
        snac_state_view v = {0};
        v.plastic_strain = self->plasticStrain;
        v.viscosity = self->viscosity;
        v.plastic_strain_tensor = self->plasticStrainTensor;
        if (v.plastic_strain || v.viscosity) cuda_check(context, self, snac_gpu_upload(self->gpu, &v), "snac_gpu_upload");
    }
    cuda_check(context, self, snac_gpu_time_step_zero(self->gpu), "snac_gpu_time_step_zero");
    scalars_to_context(context, self);
    context->initMinLengthScale = context->minLengthScale;
}

/* Prepended to AbstractContext_EP_Solve: the device's timeStep++ and the
 * step's dt (AbstractContext.c:874-890). */
void SnacCuda_BeginStep(void* context) {
    SnacCuda_Context* self = cuda_of(context);
    cuda_check(context, self, snac_gpu_begin_step(self->gpu), "snac_gpu_begin_step");
}

void SnacCuda_LoopElementsEnergy(void* context) {
    SnacCuda_Context* self = cuda_of(context);
    cuda_check(context, self, snac_gpu_loop_elements_energy(self->gpu), "snac_gpu_loop_elements_energy");
}

void SnacCuda_LoopNodesEnergy(void* context) {
    SnacCuda_Context* self = cuda_of(context);
    cuda_check(context, self, snac_gpu_loop_nodes_energy(self->gpu), "snac_gpu_loop_nodes_energy");
}

void SnacCuda_CalcStresses(void* context) {
    SnacCuda_Context* self = cuda_of(context);
    cuda_check(context, self, snac_gpu_calc_stresses(self->gpu), "snac_gpu_calc_stresses");
}

void SnacCuda_LoopNodesMomentum(void* context) {
    SnacCuda_Context* self = cuda_of(context);
    cuda_check(context, self, snac_gpu_loop_nodes_momentum(self->gpu), "snac_gpu_loop_nodes_momentum");
}

void SnacCuda_LoopElementsMomentum(void* context) {
    SnacCuda_Context* self = cuda_of(context);
    cuda_check(context, self, snac_gpu_loop_elements_momentum(self->gpu), "snac_gpu_loop_elements_momentum");
}

/* Replaces "SnacSync" (Context.c:1208-1268) */
void SnacCuda_Sync(void* context) {
    SnacCuda_Context* self = cuda_of(context);
    cuda_check(context, self, snac_gpu_sync(self->gpu), "snac_gpu_sync");
    scalars_to_context((Snac_Context*)context, self);
}

/* device -> context: prepended to AbstractContext_EP_Dump, and for any host
 * plugin that reads the state (the remesher) */
void SnacCuda_SyncHost(void* context) {
    SnacCuda_Context* self = cuda_of(context);
    snac_state_view v;
    if (!self->gpu) return;
    v.coord = self->coord;
    v.velocity = self->velocity;
    v.stress = self->stress;
    v.plastic_strain = self->plasticStrain;
    v.viscosity = self->viscosity;
    v.temperature = self->temperature_;
    v.force = self->force;
    v.inertial_mass = self->inertialMass;
    v.plastic_strain_tensor = self->plasticStrainTensor;
    cuda_check(context, self, snac_gpu_download(self->gpu, &v), "snac_gpu_download");
    SnacCuda_Unpack((Snac_Context*)context, self);
}

/* context -> device, after a host plugin changed the state */
void SnacCuda_SyncDevice(void* context) {
    SnacCuda_Context* self = cuda_of(context);
    snac_state_view v = {0};
    if (!self->gpu) return;
    SnacCuda_Pack((Snac_Context*)context, self);
    v.coord = self->coord;
    v.velocity = self->velocity;
    v.stress = self->stress;
    v.plastic_strain = self->plasticStrain;
    v.viscosity = self->viscosity;
    v.temperature = self->temperature_;
    v.plastic_strain_tensor = self->plasticStrainTensor;
    cuda_check(context, self, snac_gpu_upload(self->gpu, &v), "snac_gpu_upload");
}

void _SnacCuda_Construct(void* component, Stg_ComponentFactory* cf, void* data) {
    Snac_Context* context;
    EntryPoint* energyEP;
    (void)component;

    context = (Snac_Context*)Stg_ComponentFactory_ConstructByName(cf, "context", Snac_Context, True, data);

    /* Add the plugin's context extension (zeroed: no device model yet) */
    SnacCuda_ContextHandle = ExtensionManager_Add(context->extensionMgr, SnacCuda_Type, sizeof(SnacCuda_Context));
    memset(cuda_of(context), 0, sizeof(SnacCuda_Context));

    /* Step zero, then the hot loop's entry points, on the device */
    EntryPoint_Replace(Context_GetEntryPoint(context, AbstractContext_EP_Initialise), "SnacTimeStepZero",
                       SnacCuda_Type, SnacCuda_TimeStepZero, SnacCuda_Type);
    EntryPoint_Prepend(Context_GetEntryPoint(context, AbstractContext_EP_Solve), "SnacCuda_BeginStep",
                       SnacCuda_BeginStep, SnacCuda_Type);
    EntryPoint_Replace(Context_GetEntryPoint(context, Snac_EP_CalcStresses), "default", SnacCuda_Type,
                       SnacCuda_CalcStresses, SnacCuda_Type);
    EntryPoint_Replace(Context_GetEntryPoint(context, Snac_EP_LoopNodesMomentum), "default", SnacCuda_Type,
                       SnacCuda_LoopNodesMomentum, SnacCuda_Type);
    EntryPoint_Replace(Context_GetEntryPoint(context, Snac_EP_LoopElementsMomentum), "default", SnacCuda_Type,
                       SnacCuda_LoopElementsMomentum, SnacCuda_Type);
    EntryPoint_Replace(Context_GetEntryPoint(context, AbstractContext_EP_Sync), "SnacSync", SnacCuda_Type,
                       SnacCuda_Sync, SnacCuda_Type);

    /* The temperature plugin's energy loops, when it is loaded (it must come
     * before SnacCuda in the import list) */
    energyEP = Context_GetEntryPoint(context, Snac_EP_LoopElementsEnergy);
    if (energyEP && energyEP->hooks->count)
        EntryPoint_ReplaceAll(energyEP, SnacCuda_Type, SnacCuda_LoopElementsEnergy, SnacCuda_Type);
    energyEP = Context_GetEntryPoint(context, Snac_EP_LoopNodesEnergy);
    if (energyEP && energyEP->hooks->count)
        EntryPoint_ReplaceAll(energyEP, SnacCuda_Type, SnacCuda_LoopNodesEnergy, SnacCuda_Type);

    /* The dump hooks (the reference's writers) read the context: bring it up to date first */
    EntryPoint_Prepend(Context_GetEntryPoint(context, AbstractContext_EP_Dump), "SnacCuda_SyncHost",
                       SnacCuda_SyncHost, SnacCuda_Type);
}
