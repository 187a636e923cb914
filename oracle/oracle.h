// oracle.h -- TEST INFRASTRUCTURE ONLY.  C interface of the CPU oracle (a
// restatement of the reference's per-stage hot path, slug-cfd/kfvm-kokkos).
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
#ifndef KFVM_ORACLE_H_
#define KFVM_ORACLE_H_

#include <stdint.h>

#include "../include/kfvm_b200.h"

#ifdef __cplusplus
namespace orc {
void quad_rule(int nq, double *ab, double *wt);
int build_stencil(const kfvm_config *cfg, kfvm_stencil *st);
} // namespace orc
extern "C" {
#endif

typedef struct orc_solver orc_solver;

int orc_stencil_build(const kfvm_config *cfg, kfvm_stencil *out);
orc_solver *orc_create(const kfvm_config *cfg);
void orc_destroy(orc_solver *s);
int orc_set_threads(int n);
int orc_init_ic(orc_solver *s, int32_t ic_kind, uint64_t seed);
int orc_set_state(orc_solver *s, const double *u);
int orc_get_state(orc_solver *s, double *u);
int orc_eval_rhs(orc_solver *s, double t, double *rhs, double *max_vel);
int orc_take_step(orc_solver *s, kfvm_step_info *info);
int orc_solve(orc_solver *s, int32_t max_steps, int64_t *n_steps, kfvm_step_info *last);
int orc_get_time(orc_solver *s, double *time, double *dt);
int orc_set_time(orc_solver *s, double time, double dt);
/* Flow statistics of the current state (n_stats = 2, GLM-MHD 3, SRHydro 1). */
int orc_flow_stats(orc_solver *s, double *stats, int32_t *n_stats);
/* Random forcing with a given mode table (n_modes x dim x 3). */
int orc_apply_forcing(orc_solver *s, const double *modes, int32_t n_modes, double edot, double ratio,
                      double *force_str);
/* Keep a copy of the face states before the Riemann solve for orc_get_faces. */
int orc_keep_faces(orc_solver *s, int32_t on);
int orc_get_faces(orc_solver *s, int32_t dir, double *out);
int orc_get_flags(orc_solver *s, uint8_t *weno_applied, double *theta);
int orc_weno_departure(orc_solver *s, double *out);
int orc_set_indicator(orc_solver *s, int32_t ind);
/* Domain decomposition: cfg->nb and cfg->block place this solver's block in the
 * whole domain (kfvm_block_config makes such a configuration); its
 * KFVM_BC_EXCHANGE faces take their halo cells and outer face states from the
 * neighbouring ranks through ex, and the maxima, sums and minima of a step go
 * through ar, with the meaning of kfvm_set_exchange's callbacks on host buffers. */
int orc_set_exchange(orc_solver *s, kfvm_exchange_fn ex, kfvm_allreduce_fn ar, void *user);
/* User boundary conditions: KFVM_BC_USER faces call fn with host buffers, with
 * the meaning and layouts of kfvm_set_user_bc (stream NULL). */
int orc_set_user_bc(orc_solver *s, kfvm_user_bc_fn fn, void *user);
/* Quadrature and RK coefficient tables used by the oracle. */
int orc_tables(int32_t nq, int32_t rk, double *quad, double *rkt);
/* Initial-condition cell averages alone (no FSAL priming), SoA interior. */
int orc_ic_cells(const kfvm_config *cfg, int32_t ic_kind, uint64_t seed, double *u);

#ifdef __cplusplus
}
#endif

#endif
