/*
 * gd_oracle.h -- CPU restatement of the reference swarm collision path.
 *
 * TEST INFRASTRUCTURE ONLY.  This oracle is the checker for libgd_b200: only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline / reference arm may load it.  The product
 * never calls it and has no CPU fallback.
 *
 * Each function cites the reference file:line it restates (paths inside the GameDev tree).
 * Floating-point policy: single-precision distances use the fmaf chain pinned in the CUDA
 * kernels (compiled with -ffp-contract=off so no other contraction happens); FP64 physics uses
 * libm, so it agrees with the GPU to a few ulps, not bit for bit.
 */
#ifndef GD_ORACLE_H
#define GD_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#include "../include/gd_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* col_site_init (src/swarm/col_site_init.cu:17-55): sites [n][4] = (x, y, z, code bits),
 * search radius q[n] (0 when inactive), active[n].  Returns the smallest non-finite index or -1. */
int gdo_site_init(const gd_config *cfg, const gd_particle *p, int n, float *site4, float *q, unsigned char *active);

/* Exact top-K of every active owner among active sites with d^2 <= q_i^2, keyed by
 * (float d^2 bits << 32 | code) as in kdtree/index_heap.cuh:58-69, written ascending.
 * codes[n][K] (-1 padding, inactive rows all -1), d2[n][K] (may be NULL).
 * gdo_knn_brute: O(n^2) loop, the brute force of val/swarm/mod/test_knn/knn_benchmark.cu:508-548.
 * gdo_knn_kdtree: KD tree with widest-dimension median splits (the split rule of
 * kdtree/builder_thrust.h:263-318) and the reference heap; `threads` OpenMP threads. */
void gdo_knn_brute(int n, const float *site4, const float *q, const unsigned char *active, int K, int32_t *codes,
                   float *d2, int threads);
void gdo_knn_kdtree(int n, const float *site4, const float *q, const unsigned char *active, int K, int32_t *codes,
                    float *d2, int threads, int first, int count);

/* The same top-K over sites that include azimuthal-wedge images (col_site_init.cu:58-76): owners
 * are sites 0..n-1 (image 0); every one of the n_sites sites (code = 3 * particle + image) is a
 * candidate, active when its particle is.  An owner with image_dist_min <= 2 q keeps one image per
 * particle, the one with the smaller key (the dedup of kdtree/index_heap.cuh:118-141); q is the
 * owner's own q_i (KD search, _col_cache.cuh:38-39) or q_dedup >= 0 (Morton search: the largest
 * q, swarm_runtime.cu:413-415).  image_dist_min < 0: no dedup.  A site whose code is -1 is an
 * image the Morton ghost rule dropped and is no candidate. */
void gdo_knn_brute_images(int n, int n_sites, const float *site4, const float *q, const unsigned char *active,
                          int K, float image_dist_min, float q_dedup, int32_t *codes, float *d2, int threads);

/* The Morton ghost rule (morton_ghost.cuh:28-50) over n physical sites: keep[2i] for image 1
 * (-width, the x_max seam), keep[2i+1] for image 2 (+width, the x_min seam); margin[] the relative
 * distance of each decision from q_max. */
void gdo_morton_ghosts(int n, const float *site4, const float *posx, float q_max, float x_min, float x_max,
                       unsigned char *keep, double *margin);

/* The pinned single-precision squared distance. */
float gdo_dist2(const float *a, const float *b);

/* _get_ball_measure (inc/swarm/_collision.cuh:66-115) of every owner from its largest kept d^2
 * (kth_d2[i], 0 for an empty row); 0 for inactive owners. */
void gdo_ball_measure(const gd_config *cfg, const gd_particle *p, int n, const unsigned char *active,
                      const float *kth_d2, double *measure);

/* col_space_bin (src/swarm/col_space_bin.cu:11-35) */
void gdo_space_bin(const gd_config *cfg, const gd_particle *p, int n, int32_t *spatial);

/* ---- collision operator (gd_oracle_collide.c) ---- */
void   gdo_env(const gd_config *c, double y, double z, double *env8);
double gdo_pair_speed_cached(const gd_config *c, const double *env8, double size_i, double size_j);
double gdo_pair_speed_direct(const gd_config *c, double y, double z, double size_i, double size_j);
double gdo_pair_rate(const gd_config *c, double yi, double zi, double yj, double zj, double size_i, double size_j,
                     double numr_j, double lambda0, double measure, double *vrel);
double gdo_outcome_moments(const gd_config *c, double si, double sj, int high, double *mean_second_max);
double gdo_sample_outcome(const gd_config *c, double si, double sj, int high, double u);
void   gdo_bath_rate(const gd_config *c, int n, const gd_particle *p, const int32_t *codes, const double *measure,
                     const unsigned char *active, const double *size_old, const double *numr_old, double lambda0,
                     double *cached4, double *rate, double *change, double *second, int threads);
int    gdo_chain_owner(const gd_config *c, int i, const gd_particle *p, const int32_t *codes,
                       const double *measure, const unsigned char *active, const double *size_old,
                       const double *numr_old, double lambda0, double bath_end, const double *cached4,
                       const double *u, int nu, double *state8, int *used);

#ifdef __cplusplus
}
#endif

#endif
