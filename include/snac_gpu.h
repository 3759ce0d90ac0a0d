/*
 * snac_gpu.h — C ABI of the B200 (sm_100a) implementation of SNAC's explicit
 * Lagrangian time step (FLAC dynamic relaxation on a structured hex mesh,
 * each hex split into two overlapping sets of five tetrahedra).
 *
 * Plain C: pointers, sizes and integer status codes only.  Every entry point
 * returns SNAC_GPU_OK (0) or a negative SNAC_GPU_E* code; the message and the
 * offending element/node id are kept per handle (snac_gpu_last_error /
 * snac_gpu_error_index).  One handle owns one CUDA stream; a handle is
 * single-threaded and non-reentrant, like the Snac_Context it stands in for
 * (Snac/libSnac/src/Tetrahedra.c:30 notes the reference is not thread-safe).
 *
 * Conventions (Snac/libSnac/src/Context.c, StGermain HexaEL/BlockGeometry):
 *   nx, ny, nz     element (hex) counts along I (x), J (y, vertical, gravity
 *                  acts on -y) and K (z).  Node counts are nx+1, ny+1, nz+1
 *                  (the reference's meshSizeI/J/K).
 *   node (i,j,k)   index i + j*(nx+1) + k*(nx+1)*(ny+1)
 *   element (i,j,k) index i + j*nx + k*nx*ny
 *   tensors        6 components per tetrahedron in the order
 *                  xx, yy, zz, xy, xz, yz (upper triangle of the reference's
 *                  3x3 arrays; the lower triangle is never written there).
 *   host arrays    element-major: stress[((e*10)+t)*6 + c],
 *                  plastic_strain[e*10 + t], coord/velocity[n*3 + d].
 */
#ifndef SNAC_GPU_H
#define SNAC_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SNAC_GPU_ABI_VERSION 2  /* snac_gpu_create also takes version-1 descriptors (up to topo_grad_criterion) */

/* ---- status codes ------------------------------------------------------ */
#define SNAC_GPU_OK          0
#define SNAC_GPU_EINVAL     -1   /* bad descriptor or argument                       */
#define SNAC_GPU_ENOMEM     -2   /* device or host allocation failed                 */
#define SNAC_GPU_ECUDA      -3   /* CUDA runtime error                               */
#define SNAC_GPU_ENAN       -4   /* NaN/Inf in the state (reference: Journal firewall)*/
#define SNAC_GPU_EVOLUME    -5   /* zero tetrahedron volume (degenerate element)     */
#define SNAC_GPU_EMATERIAL  -6   /* material index out of range                      */
#define SNAC_GPU_EPHYSICS   -7   /* reference abort()/assert(): friction angle < 0,
                                    dt_thermal/dt_mech <= 1, ...                      */
#define SNAC_GPU_ETIMEDOUT  -8   /* a bounded device-side wait gave up               */
#define SNAC_GPU_ENOTSUP    -9   /* option the reference has but this build does not  */
#define SNAC_GPU_ESTATE    -10   /* call out of order (e.g. step before step zero)    */
#define SNAC_GPU_ENODEV    -11   /* no CUDA device                                   */

/* ---- enumerations (values follow the reference where it has them) ------ */
/* dtType, Snac/libSnac/src/Context.c:345-391 */
#define SNAC_DT_CONSTANT 0
#define SNAC_DT_DYNAMIC  1
#define SNAC_DT_WAVE     2

/* Material rheology bits, Snac/libSnac/src/Material.h:46-50.  The
 * "constitutive" field of the descriptor names the ONE constitutive plugin
 * loaded on Snac_EP_Constitutive (SnacElastic, SnacPlastic, SnacViscoPlastic
 * or SnacMaxwell), as in the reference configs. */
#define SNAC_RHEOLOGY_ELASTIC      0x1
#define SNAC_RHEOLOGY_PLASTIC      0x2
#define SNAC_RHEOLOGY_MAXWELL      0x4
#define SNAC_RHEOLOGY_VISCOPLASTIC 0x8

/* Wall ids, StGermain/Discretisation/Utils/src/WallVC.c:49-55 */
#define SNAC_WALL_BACK   0   /* k == 0        */
#define SNAC_WALL_LEFT   1   /* i == 0        */
#define SNAC_WALL_BOTTOM 2   /* j == 0        */
#define SNAC_WALL_RIGHT  3   /* i == nx       */
#define SNAC_WALL_TOP    4   /* j == ny       */
#define SNAC_WALL_FRONT  5   /* k == nz       */
#define SNAC_WALL_ALL    6   /* every node (AllNodesVC)                          */

#define SNAC_MAX_SEGMENTS 8  /* softening table: nsegments <= 8, 9 break points */
#define SNAC_MAX_PHASES   32 /* n_materials <= 32; finer variation goes in the per-element scales */

/* One phase, Snac/libSnac/src/Material.h:54-112 and the dictionary keys of
 * Context.c:826-914.  Every value is taken as given (no float-literal
 * defaults are applied here; pass what the reference would have read). */
typedef struct snac_material {
    double density;          /* phsDensity                    */
    double alpha, beta;      /* thermal expansion, compressibility */
    double lambda, mu;
    int    nsegments;        /* piecewise-linear softening     */
    int    yield_mohr_coulomb; /* 1: mohrcoulomb; 0: druckerprager, which only the visco-plastic hook
                                  has (viscoplastic/Constitutive.c:372-518; the plastic hook always
                                  takes Mohr-Coulomb, plastic/Constitutive.c:58-247) */
    double plstrain[SNAC_MAX_SEGMENTS + 1];
    double friction_angle[SNAC_MAX_SEGMENTS + 1];   /* degrees */
    double dilation_angle[SNAC_MAX_SEGMENTS + 1];   /* degrees */
    double cohesion[SNAC_MAX_SEGMENTS + 1];
    double ten_off;
    double vis_min, vis_max, refvisc, refsrate, reftemp;
    double activation_e;     /* activationE (J/mol)            */
    double srexponent;
    double thermal_conduct, heat_capacity;
} snac_material;

/* One entry of a CompositeVC vcList (WallVC / AllNodesVC).  For velocity
 * BCs bit d of mask fixes component d to value[d]; for temperature BCs bit 0
 * fixes T to value[0].  When several entries fix the same component of the
 * same node the LAST one wins (StGermain/Base/Automation/src/CompositeVC.c:599-611). */
typedef struct snac_wall_bc {
    int    wall;
    int    mask;
    double value[3];
} snac_wall_bc;

typedef struct snac_gpu_desc {
    int    abi_version;              /* SNAC_GPU_ABI_VERSION */
    int    nx, ny, nz;
    double min[3], max[3];           /* BlockGeometry extent */
    const double* node_coords;       /* optional [nn*3]; overrides the block geometry */

    int    dt_type;                  /* SNAC_DT_*                     */
    double dt;                       /* "timeStep": constant dt, or the initial value */
    double strain_inert;
    double gravity;
    double demf;                     /* FLAC local damping factor     */

    int    constitutive;             /* one SNAC_RHEOLOGY_* bit        */
    int    temperature;              /* SnacTemperature loaded         */
    int    compute_thermal_stress;
    int    hydrostatic_ic;           /* SnacHydroStaticIC loaded       */
    int    temperature_sweep_ic;     /* _SnacTemperature_Top2BottomSweep as the node IC */
    double top_temp, bottom_temp;    /* for the sweep IC               */

    int    n_materials;
    const snac_material* materials;
    const int*    element_material;  /* [ne] phase id, NULL = 0       */
    /* Optional per-element multipliers of the phase tables: the reference
     * expresses these as one phase per element with scaled table values. */
    const double* element_cohesion_scale;  /* [ne] x cohesion[i]       */
    const double* element_friction_scale;  /* [ne] x frictionAngle[i]  */
    const double* element_visc_scale;      /* [ne] x refvisc           */

    int    n_velocity_bcs;
    const snac_wall_bc* velocity_bcs;
    int    n_temperature_bcs;
    const snac_wall_bc* temperature_bcs;

    const double* init_velocity;     /* [nn*3] nodeICs, NULL = 0      */
    const double* init_temperature;  /* [nn], used when temperature_sweep_ic == 0 */
    const double* init_stress;       /* [ne*10*6] elementICs, NULL = 0 (hydrostatic_ic adds on top) */

    /* SnacWinklerForce loaded (Snac/plugins/winkler/Force.c:56-168): bottom
     * support on the j = 0 nodes from the isostatic pressure pisos and the
     * reference bottom depth rzbo, both set by the hydrostatic IC
     * (hydroStaticIC/VariableConditions.c:120-138; 0 without it). */
    int    winkler;
    /* SnacTractionBC loaded (Snac/plugins/tractionBC/Force.c:43-268): its one
     * active branch applies the fixed stress sxx = 1e8 Pa on the right wall
     * (i = nx).  Force hooks run in load order: Winkler, then traction. */
    int    traction_bc;
    /* Surface-topography diffusion of the top nodes (UpdateNode.c:161-857,
     * cartesian geometry): "topo_kappa" (0 = off; the reference's dictionary
     * default is 5e-6) and "topoGradCriterion" (default 1e-16). */
    double topo_kappa;
    double topo_grad_criterion;

    /* ---- ABI version 2 ----
     * For a caller that ran the initial conditions itself (a Snac_Context
     * after its plugin ICs, as the SnacCuda plugin passes it): the isostatic
     * pressure and reference bottom depth SnacWinklerForce reads
     * (context->pisos, element->rzbo), used when hydrostatic_ic == 0. */
    double pisos, rzbo;
    /* Velocity and temperature conditions resolved per node, in place of
     * velocity_bcs / temperature_bcs when the mask is non-NULL: bit d of
     * node_velocity_bc_mask[n] fixes component d of node n to
     * node_velocity_bc_value[n*3+d]; node_temperature_bc_mask[n] != 0 fixes
     * the temperature to node_temperature_bc_value[n].  At most 254 distinct
     * values per velocity component and 254 temperatures (SNAC_GPU_ENOTSUP
     * beyond).  The CPU checkers under oracle/ take the wall form only. */
    const unsigned char* node_velocity_bc_mask;
    const double* node_velocity_bc_value;
    const unsigned char* node_temperature_bc_mask;
    const double* node_temperature_bc_value;
    /* Drucker-Prager phases of the visco-plastic hook: per phase "maxiterations"
     * and "constitutivetolerance" (Context.c:851-854); NULL = the reference's
     * defaults, 1 and 1e-3. */
    const int*    dp_max_iterations;
    const double* dp_tolerance;
} snac_gpu_desc;

/* Host-side view of the state for upload / download.  NULL members are
 * skipped.  Sizes: nn*3, nn*3, ne*10*6, ne*10, ne*10, nn, nn*3, nn, ne*10*6.
 * A handle created from a version-1 descriptor reads the view without its
 * last member. */
typedef struct snac_state_view {
    double* coord;
    double* velocity;
    double* stress;
    double* plastic_strain;
    double* viscosity;
    double* temperature;
    double* force;           /* download only: damped nodal force of the last step */
    double* inertial_mass;   /* download only */
    /* ABI version 2: the visco-plastic plugin's per-tet plastic strain tensor
     * (plasticstrainTensor, viscoplastic/Element.h; xx, yy, zz, xy, xz, yz),
     * [ne*10*6]; kept by models with a Drucker-Prager phase, zero otherwise. */
    double* plastic_strain_tensor;
} snac_state_view;

typedef struct snac_scalars {
    double dt;               /* dt the NEXT step will use            */
    double min_length_scale; /* global minimum of |V/A|              */
    double vmax;             /* max |v| over velocity-BC nodes (floored at 3e-11f) */
    double speed_of_sound;
    long long time_step;     /* steps completed after step zero      */
    double current_time;     /* sum of the steps' dt (AbstractContext currentTime) */
} snac_scalars;

typedef struct snac_gpu snac_gpu;

/* ---- lifetime ------------------------------------------------------------ */
/* Builds the device state from the descriptor and applies the initial
 * conditions in the reference's order: nodeICs, elementICs, velocity BCs
 * (Context.c:742-774), then the plugin ICs inserted before SnacTimeStepZero
 * (temperature, plastic / visco-plastic / Maxwell, hydrostatic).
 * Replaces Snac_Context construction + _Snac_Context_InitialConditions. */
int  snac_gpu_create(const snac_gpu_desc* desc, snac_gpu** out);
void snac_gpu_destroy(snac_gpu* h);

/* Snac_Context_TimeStepZero (Context.c:978-1036): element geometry from the
 * initial coordinates, then Sync (first dt). */
int  snac_gpu_time_step_zero(snac_gpu* h);

/* nsteps x _AbstractContext_Step (AbstractContext.c:921-941) with the SNAC
 * hooks: Solve (_Snac_Context_Solve, Context.c:1063-1099) then Sync
 * (_Snac_Context_Sync, Context.c:1208-1268).  The step loop runs from a CUDA
 * graph; nothing is copied to the host. */
int  snac_gpu_step(snac_gpu* h, int nsteps);
/* Measurement helper (no counterpart in the reference): nsteps steps as in
 * snac_gpu_step, each preceded on the handle's stream by a write of
 * flush_bytes to flush (NULL / 0: none; a buffer larger than L2 evicts the
 * model state), and bracketed by CUDA events; ms[i] receives the device time
 * of step i alone.  The status is read once, after all steps. */
int  snac_gpu_time_steps(snac_gpu* h, int nsteps, void* flush, size_t flush_bytes, double* ms);

/* Loop-level entry points, one per StGermain entry point a plugin replaces
 * with EntryPoint_Replace (StGermain/Base/Extensibility/src/EntryPoint.c:735):
 *   Snac_EP_LoopElementsEnergy   (temperature/HeatFlux.c:47-58)
 *   Snac_EP_LoopNodesEnergy      (temperature/Heat.c:47-62)
 *   Snac_EP_CalcStresses         (_Snac_Context_CalcStresses, Context.c:1102-1117)
 *   Snac_EP_LoopNodesMomentum    (_Snac_Context_LoopNodes, Context.c:1120-1154)
 *   Snac_EP_LoopElementsMomentum (_Snac_Context_LoopElements, Context.c:1156-1184)
 *   AbstractContext_EP_Sync      (_Snac_Context_Sync, Context.c:1208-1268)
 * snac_gpu_begin_step advances timeStep and takes dt for the step the way
 * _AbstractContext_Execute_Hook / _Snac_Context_Dt do (AbstractContext.c:874-890). */
int  snac_gpu_begin_step(snac_gpu* h);
int  snac_gpu_loop_elements_energy(snac_gpu* h);
int  snac_gpu_loop_nodes_energy(snac_gpu* h);
int  snac_gpu_calc_stresses(snac_gpu* h);
int  snac_gpu_loop_nodes_momentum(snac_gpu* h);
int  snac_gpu_loop_elements_momentum(snac_gpu* h);
int  snac_gpu_sync(snac_gpu* h);

/* ---- state transfer -------------------------------------------------------- */
int  snac_gpu_upload(snac_gpu* h, const snac_state_view* v);
int  snac_gpu_download(snac_gpu* h, const snac_state_view* v);
/* One step of a model whose state the host keeps: the fields `in` names are
 * uploaded, one step runs (snac_gpu_step), and the fields `out` names are
 * downloaded; the result has the bits of snac_gpu_upload(in) +
 * snac_gpu_step(h, 1) + snac_gpu_download(out).  Replaces, for a host that
 * owns the Snac context's arrays between steps, the per-step transfers
 * around _Snac_Context_Solve (Context.c:1063-1099) and Sync (:1208-1268).
 *   - The transfers overlap the kernels and each other: the mesh is cut
 *     along k into `chunks` slabs (at most 64; 0: one per 6 MiB of tet
 *     stresses, 1 to 16); each slab's kernels
 *     start when its upload has arrived, and its download starts when its
 *     last kernel is done.  The overlap needs page-locked host arrays
 *     (cudaHostAlloc / cudaHostRegister); pageable ones give the same
 *     result without it.
 *   - `in` and `out` may name the same arrays (the step updates them in
 *     place); NULL members are not transferred.
 *   - Models with topography diffusion or open dump files, or an `out`
 *     asking for force or inertial mass, run the three calls in sequence.
 *   - Device memory: node staging of 14 doubles per node, allocated on the
 *     first call, with two streams and the slab events. */
int  snac_gpu_step_host(snac_gpu* h, const snac_state_view* in, const snac_state_view* out, int chunks);
int  snac_gpu_scalars(snac_gpu* h, snac_scalars* out);
int  snac_gpu_set_dt(snac_gpu* h, double dt);   /* _Snac_Context_SetDt, Context.c:1047-1053 */

/* ---- dump and checkpoint files --------------------------------------------------
 * The reference's output files (Snac/libSnac/src/Context.c:1311-1531 with
 * StGermain's VariableDumpStream, the plastic / visco-plastic / temperature
 * plugins' Output.c): raw float32 records (int32 phase indices) appended per
 * dump or checkpoint step to <output_path>/<name>.<rank>:
 *   dump:       strainRate, stress, hydroPressure (element scalars), phaseIndex,
 *               coord, vel, force (3 per node), stressTensor (6 per element,
 *               volume-weighted in float), plStrain (aps), viscosity (log10 of
 *               the mean), temperature
 *   checkpoint: phaseIndexCP, coordCP, velCP, stressTensorCP (6 per tet),
 *               plStrainCP, viscosityCP (log10 per tet), temperatureCP
 *   rank 0:     sim.0, and timeStep.0 / checkpointTimeStep.0 lines
 *               "%16u %16g %16g" (timeStep, currentTime, dt).
 * Open before stepping: the steps whose end is a dump (isTimeToDump:
 * timeStep 1 and every dump_every) then also store the element scalars.
 * snac_gpu_write_output is _Snac_Context_WriteOutput + the loop-info writers
 * for the current timeStep; it packs the records on the device, copies them
 * into pinned memory and returns, and a writer thread appends them to the
 * files (the next write or close waits for it). */
int  snac_gpu_output_open(snac_gpu* h, const char* output_path, unsigned rank, unsigned dump_every,
                          unsigned checkpoint_every, unsigned max_time_steps);
int  snac_gpu_write_output(snac_gpu* h);
int  snac_gpu_output_close(snac_gpu* h);

/* ---- profiling ---------------------------------------------------------------- */
/* One step launched kernel by kernel (no graph), with CUDA events recorded
 * around every launch on the handle's stream: names[i] / ms[i] for the
 * kernels of the step, in launch order.  Returns the number of kernels
 * (<= max) or a negative status.  The step advances the model like
 * snac_gpu_step(h, 1). */
typedef struct snac_kernel_time {
    char   name[40];
    double ms;
} snac_kernel_time;
int  snac_gpu_profile_step(snac_gpu* h, snac_kernel_time* out, int max);

/* Node fields (coord[nn*3], velocity[nn*3], temperature[nn]; any may be
 * NULL) copied to host arrays like snac_gpu_download, but without allocating
 * anything: no cudaMalloc/cudaFree, no library allocator.  For callers that
 * must not allocate device memory during a run, e.g. a dump hook of a
 * process whose device memory is fully committed to its models, where the
 * lazily allocated staging buffer of snac_gpu_download could fail or evict.
 * No counterpart in the reference (its node arrays are host memory).
 *   - Staging is a static device array of 262,144 nodes x 3 doubles
 *     (6 MiB); models with more nodes get SNAC_GPU_EINVAL and a message.
 *   - Nothing in the staging has to start at zero: each call writes every
 *     staged value before copying it out.
 *   - The first call on each device looks up the staging address
 *     (cudaGetSymbolAddress) with that device current and keeps it for the
 *     life of the process; make that first call before any stream capture
 *     begins.  The handle's device must be current.  A cudaDeviceReset
 *     invalidates that address together with every handle on the device:
 *     after one, this library must not be used again in the process.
 *   - snac_gpu_device_bytes of the handle does not change across the call.
 *   - One staging array per device: overlapping calls would race on it, so
 *     the call holds a process-wide lock until its copies have finished
 *     (calls from several threads run one after another).
 * Applies a pending element update first, as snac_gpu_download does. */
int  snac_gpu_download_nodes_noalloc(snac_gpu* h, double* coord, double* velocity, double* temperature);

/* ---- errors / introspection ------------------------------------------------ */
const char* snac_gpu_last_error(const snac_gpu* h);
long long   snac_gpu_error_index(const snac_gpu* h);   /* element/node id, -1 if none */
int  snac_gpu_sizes(const snac_gpu* h, long long* n_elements, long long* n_nodes);
/* Number of kernels this library launched on the handle since creation. */
long long snac_gpu_launch_count(const snac_gpu* h);
/* Device memory the library has allocated for this handle since creation,
 * in bytes (model state, lazily allocated staging, output and adjoint
 * buffers); it never decreases before snac_gpu_destroy. */
int  snac_gpu_device_bytes(const snac_gpu* h, long long* bytes);
/* The handle's cudaStream_t, as a void* (for event timing by callers). */
void* snac_gpu_stream(snac_gpu* h);
int  snac_gpu_device_count(void);
/* Measurement helper (no counterpart in the reference): the current
 * device's FP64 throughput, in fused multiply-adds per second (one FP64
 * instruction per thread each), from independent FMA chains over a grid of
 * 8 blocks per SM; the best of three timed launches after a warm-up.  The
 * FP64 roofline of a kernel is its FP64 instructions per second against
 * this rate. */
int  snac_gpu_fp64_rate(double* fma_per_second);
/* Self-test of the straight-line correctly rounded division the kernels use
 * (csrc/snac_device.cuh): n random operand pairs (wide exponent range,
 * signed zeros, exact quotients and ties) compared bit for bit with the
 * IEEE quotient of the GPU; *mismatches receives the count (expected 0). */
int  snac_gpu_selftest_division(long long n, unsigned long long seed, long long* mismatches);

/* ---- adjoint ------------------------------------------------------------------
 * No counterpart in the reference.  Loss on the top surface (node plane
 * j = ny, node order i + k*(nx+1)) after nsteps steps from the current state:
 *   L = sum w_v (v_y - target_vy)^2 + w_h (y - target_y)^2
 * snac_gpu_adjoint runs the nsteps forward (keeping every checkpoint_every-th
 * state; 0 = ceil(sqrt(nsteps))), then the hand-written reverse sweep
 * segment by segment (each segment recomputed from its checkpoint), and
 * returns L and dL/d(scale) for the per-element cohesion, friction-angle
 * and viscosity scales (element_cohesion_scale / element_friction_scale /
 * element_visc_scale; an absent array is a scale of 1).  On return the model
 * holds the forward's final state, as after snac_gpu_step(h, nsteps).
 * Differentiated physics: the SnacElastic, SnacMaxwell, SnacPlastic and
 * SnacViscoPlastic hooks (Mohr-Coulomb return map along the branch the
 * forward took), dtType constant, no density coupling or thermal stress,
 * temperature held fixed (thermal_conduct = 0); otherwise SNAC_GPU_ENOTSUP.
 * (The parameter gradients of the elastic and Maxwell hooks are zero: no
 * scale enters them; snac_gpu_adjoint_grads also returns the gradients with
 * respect to the initial state.) */
typedef struct snac_adjoint_desc {
    int nsteps;
    int checkpoint_every;
    const double* target_vy;   /* [(nx+1)*(nz+1)] */
    const double* target_y;    /* [(nx+1)*(nz+1)] */
    double w_v, w_h;
} snac_adjoint_desc;

typedef struct snac_adjoint_stats {
    double ms_forward;   /* the first forward sweep (device time)                   */
    double ms_reverse;   /* segment recomputation + reverse sweep (device time)     */
    int checkpoint_every;
    int checkpoints;
} snac_adjoint_stats;

int  snac_gpu_adjoint(snac_gpu* h, const snac_adjoint_desc* a, double* loss, double* grad_cohesion,
                      double* grad_friction, double* grad_viscosity, snac_adjoint_stats* stats);
/* The same sweep, returning any subset of dL/d(scale) and of the gradients
 * with respect to the state the model held on entry: coordinates and
 * velocities (node order, 3 per node), the tet stresses and plastic
 * strains (element-major, as the state view lays them out).  The state
 * gradients hold every other state entry fixed; for the Maxwell hook that
 * includes the stored tet volumes the first step's volume ratio reads.
 * A null pointer skips that output. */
typedef struct snac_adjoint_grads {
    double* cohesion;        /* [ne]        */
    double* friction;        /* [ne]        */
    double* viscosity;       /* [ne]        */
    double* coordinates;     /* [nn*3]      */
    double* velocity;        /* [nn*3]      */
    double* stress;          /* [ne*10*6]   */
    double* plastic_strain;  /* [ne*10]     */
} snac_adjoint_grads;
int  snac_gpu_adjoint_grads(snac_gpu* h, const snac_adjoint_desc* a, double* loss, const snac_adjoint_grads* g,
                            snac_adjoint_stats* stats);
/* L of the current state (no stepping): the forward half of the above, for
 * finite-difference checks. */
int  snac_gpu_misfit(snac_gpu* h, const snac_adjoint_desc* a, double* loss);

/* ---- batched ensembles ------------------------------------------------------
 * No counterpart in the reference, which runs one model per process (one
 * Snac_Context per MPI job).  A batch holds n independent models, each built
 * from its own descriptor exactly as snac_gpu_create builds it (uneven mesh
 * sizes, rheologies and materials allowed), and advances all of them with ONE
 * launch per kernel type per step: each launch walks a list of work tiles
 * (model, block) over every model, and the step loop runs from CUDA graphs.
 * Per-model results are bit-identical to stepping each model on its own.
 * The models share one CUDA stream; snac_gpu_batch_model() returns a model's
 * handle, through which state is downloaded or uploaded and scalars read
 * (those calls are stream-ordered with the batch's steps). */
typedef struct snac_gpu_batch snac_gpu_batch;

typedef struct snac_batch_tuning {
    int node_threads;       /* threads per node tile (64, 128, 256): nodes per tile        */
    int minls_threads;      /* threads per min-length-scale tile (64, 128, 256)            */
    int elem_blocks_per_sm; /* element launches: 0 = one block per tile, k > 0 = a
                               persistent grid of k x SMs blocks striding over the tiles */
    int node_blocks_per_sm; /* the same for the node launches                                */
    int steps_per_graph;    /* steps captured in one CUDA graph (1..256)                     */
    int order;              /* tile order: 0 = largest model first, 1 = model order          */
    int split_classes;      /* 1: one element launch per rheology class present (specialised
                               kernels), 0: one launch with a run-time switch               */
} snac_batch_tuning;

int  snac_gpu_batch_create(const snac_gpu_desc* descs, int n_models, snac_gpu_batch** out);
void snac_gpu_batch_destroy(snac_gpu_batch* b);
/* Snac_Context_TimeStepZero of every model. */
int  snac_gpu_batch_time_step_zero(snac_gpu_batch* b);
/* nsteps steps of every model, one launch per kernel type per step. */
int  snac_gpu_batch_step(snac_gpu_batch* b, int nsteps);
/* The same nsteps steps, model after model, each model's step with its own
 * launches (its snac_gpu_step graph) on the shared stream: the
 * one-launch-per-model baseline the batched form is measured against. */
int  snac_gpu_batch_step_each(snac_gpu_batch* b, int nsteps);
snac_gpu* snac_gpu_batch_model(snac_gpu_batch* b, int i);
int  snac_gpu_batch_size(const snac_gpu_batch* b);
int  snac_gpu_batch_get_tuning(const snac_gpu_batch* b, snac_batch_tuning* out);
/* Applies a launch shape (validated; SNAC_GPU_EINVAL if out of range). */
int  snac_gpu_batch_set_tuning(snac_gpu_batch* b, const snac_batch_tuning* t);
/* Runs nsteps batched steps and returns their device time in *ms (CUDA
 * events on the batch stream around the launches): the autotuner's probe. */
int  snac_gpu_batch_time_steps(snac_gpu_batch* b, int nsteps, int each, double* ms);
const char* snac_gpu_batch_last_error(const snac_gpu_batch* b);
int  snac_gpu_batch_error_model(const snac_gpu_batch* b);  /* model of the last error, -1 if none */
long long snac_gpu_batch_launch_count(const snac_gpu_batch* b);
void* snac_gpu_batch_stream(snac_gpu_batch* b);

#ifdef __cplusplus
}
#endif
#endif /* SNAC_GPU_H */
