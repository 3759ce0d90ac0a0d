/*
 * snac_oracle.h — CPU restatement of SNAC's explicit Lagrangian step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the CUDA path is compared
 * against; only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg may load it.  The product library (snac_b200) never links or calls it.
 *
 * It takes the product's descriptor (include/snac_gpu.h) so that both sides
 * are configured from one struct, and restates, in plain C with the
 * reference's operation order, Snac/libSnac/src/{Tetrahedra,UpdateElement,
 * StrainRate,Stress,Force,UpdateNode,Context}.c and the constitutive /
 * energy hooks of Snac/plugins/{elastic,plastic,viscoplastic,maxwell,
 * temperature,hydroStaticIC}.  Parity of this restatement is pinned against
 * the reference's own sources compiled here (oracle/Makefile -> oracle/_ref)
 * and against the reference's golden files (tests/golden).
 */
#ifndef SNAC_ORACLE_H
#define SNAC_ORACLE_H

#include "../include/snac_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct so_ctx so_ctx;

so_ctx* so_create(const snac_gpu_desc* d, int* status);
void    so_destroy(so_ctx* s);
int     so_time_step_zero(so_ctx* s);
int     so_step(so_ctx* s, int nsteps);

/* the loop-level hooks, in _Snac_Context_Solve order */
int so_begin_step(so_ctx* s);
int so_loop_elements_energy(so_ctx* s);
int so_loop_nodes_energy(so_ctx* s);
int so_calc_stresses(so_ctx* s);
int so_loop_nodes_momentum(so_ctx* s);
int so_node_forces(so_ctx* s);   /* force loop only, no node update */
int so_loop_elements_momentum(so_ctx* s);
int so_sync(so_ctx* s);

int  so_get_state(so_ctx* s, const snac_state_view* v);
int  so_set_state(so_ctx* s, const snac_state_view* v);
void so_scalars(so_ctx* s, snac_scalars* out);
void so_set_dt(so_ctx* s, double dt);
const char* so_last_error(so_ctx* s);

/* per-tet geometry of the last element update: volume [ne*10],
 * area [ne*10*4], normal [ne*10*4*3]; element scalars [ne] */
void so_get_geometry(so_ctx* s, double* volume, double* area, double* normal);
void so_get_element_scalars(so_ctx* s, double* volume, double* strain_rate,
                            double* stress, double* hydro_pressure,
                            double* aps, double* min_length_scale);
void so_get_tet_fields(so_ctx* s, double* strain_rate, double* strain,
                       double* density, double* avg_temp);
void so_get_node_fields(so_ctx* s, double* mass, double* balance);

/* Tetrahedra.c:44-113, for the reference's unit-cube known answers */
double so_tetrahedra_volume(const double* c1, const double* c2, const double* c3, const double* c4);
double so_tetrahedra_surface_area(const double* c1, const double* c2, const double* c3);
void   so_tetrahedra_surface_normal(const double* c1, const double* c2, const double* c3, double* n);

/* principal stresses (plastic/Constitutive.c:249-410) of one tensor
 * (xx,yy,zz,xy,xz,yz) -> ascending s[3], directions cn[3][3] (row k = vector k) */
void so_principal_stresses(const double* stress6, double* s, double* cn);

#ifdef __cplusplus
}
#endif
#endif
