/*
 * gd_b200_controller.h -- host-side bath controller of the collision operator, exported so a
 * bridge (or a test) can drive it without a GPU.  These are the pieces the reference keeps in
 * host C++ inside its operator: inc/swarm/_col_bound.cuh (size-bin merging, bath duration,
 * post-bath audit) and inc/swarm/_col_sched.cuh (power-of-two group scheduler).
 * None of these calls touches a device.
 */
#ifndef GD_B200_CONTROLLER_H
#define GD_B200_CONTROLLER_H

#include "gd_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* _build_col_binmap (_col_bound.cuh:232-285): merge adjacent sparse size bins inside every spatial
 * group.  raw[groups*bins] counts -> out[groups*bins] merged ids; returns the merged count. */
int gd_ctl_binmap(int groups, int bins, int bin_min, const int *raw, int *out);

/* _choose_col_bath (_col_bound.cuh:288-310).  bins[n][6] = mass, weighted_rate, weighted_change,
 * weighted_second, owner_count, invalid_count.  *binding = 0 horizon, 1 mean change, 2 fluctuation. */
gd_status gd_ctl_choose_bath(const gd_config *cfg, const double *bins, int n, double remaining,
                             double limit_scale, double *out, int *binding);

/* _finish_col_bath (_col_bound.cuh:313-403).  audit[n][15] in col_audit_accum field order
 * (mass, predicted_f, predicted_e, predicted_var_f, predicted_var_e, predicted_g, predicted_var_g,
 * maximum_weight, maximum_g_jump, touched, event_weight, growth, end_mass, owner_count,
 * invalid_count); state[4] = limit_scale, activity_streak, quiet_streak, floor_streak (in/out);
 * result[10] = max_f, max_e, max_touched, max_events, max_g, max_g_upper, d_bath,
 * activity_overshoot, distribution_overshoot, persistent_overshoot. */
gd_status gd_ctl_finish_bath(const gd_config *cfg, const double *audit, int n, double *state, double *result);

/* local_schedule (_col_sched.cuh:17-183) on the 2^52-tick lattice.  edges: n rows of (n+31)/32
 * words, bit d of row c set when an owner of group c has a neighbour in group d. */
typedef struct gd_schedule gd_schedule;
gd_schedule *gd_ctl_schedule_create(double horizon, const double *requested, int n, const unsigned *edges,
                                    gd_status *status);
void gd_ctl_schedule_destroy(gd_schedule *s);
unsigned long long gd_ctl_schedule_time(const gd_schedule *s);
unsigned long long gd_ctl_schedule_end(const gd_schedule *s);
int gd_ctl_schedule_due(const gd_schedule *s, unsigned long long tick, int *groups);
gd_status gd_ctl_schedule_adapt(gd_schedule *s, unsigned long long tick, const int *groups, int n_groups,
                                const double *requested, const int *passed);
void gd_ctl_schedule_advance(gd_schedule *s, const int *groups, int n_groups);
void gd_ctl_schedule_levels(const gd_schedule *s, int *levels);

#ifdef __cplusplus
}
#endif

#endif /* GD_B200_CONTROLLER_H */
