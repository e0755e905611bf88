/*
 * gd_oracle.c -- CPU restatement of the reference's geometry stage (test infrastructure only;
 * see gd_oracle.h).  Compiled with -ffp-contract=off.
 */
#include "gd_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ---------------------------------------------------------------------------------------------
 * col_site_init (src/swarm/col_site_init.cu:17-55)
 * ------------------------------------------------------------------------------------------- */

/* _is_particle_active (inc/swarm/_transport.cuh:37-48) */
static int site_active(const gd_config *c, double y, double z) {
    if (y < c->y_min || y >= c->y_max) return 0;
    if (c->n_z > 1) {
        if (c->half_disk) {
            if (z < c->z_min || z > c->z_max) return 0;
        } else {
            if (z < c->z_min || z >= c->z_max) return 0;
        }
    }
    return 1;
}

static double cyl_R(const gd_config *c, double y, double z) { return (c->n_z > 1) ? y * sin(z) : y; }
static double cyl_Z(const gd_config *c, double y, double z) { return (c->n_z > 1) ? y * cos(z) : 0.0; }
/* _get_hg (inc/swarm/param_phys.cuh:70-72) */
static double get_hg(const gd_config *c, double R) { return c->aspr_0 * pow(R / c->R_0, 0.5 * (c->idx_q + 1.0)); }

int gdo_site_init(const gd_config *c, const gd_particle *p, int n, float *site4, float *q, unsigned char *active) {
    int bad = -1;
    for (int i = 0; i < n; ++i) {
        const double *v = &p[i].position[0];
        int finite = 1;
        for (int k = 0; k < 8; ++k) finite = finite && isfinite(v[k]);
        int32_t code = 3 * i;
        float s[4] = {0.f, 0.f, 0.f, 0.f};
        memcpy(&s[3], &code, 4);
        q[i] = 0.f;
        active[i] = 0;
        if (!finite) {
            if (bad < 0) bad = i;
            memcpy(site4 + 4 * (size_t)i, s, sizeof(s));
            continue;
        }
        double x = p[i].position[0], y = p[i].position[1], z = p[i].position[2];
        int act = site_active(c, y, z);
        double R = cyl_R(c, y, z);
        double Z = cyl_Z(c, y, z);
        if (c->n_x == 1 && c->n_z == 1) {
            s[0] = (float)R;
        } else {
            s[0] = (float)(R * cos(x));
            s[1] = (float)(R * sin(x));
            s[2] = (float)Z;
        }
        memcpy(site4 + 4 * (size_t)i, s, sizeof(s));
        active[i] = (unsigned char)act;
        if (act) q[i] = (float)(c->h_search * get_hg(c, R) * R);
    }
    return bad;
}

/* ---------------------------------------------------------------------------------------------
 * exact top-K with the reference key (kdtree/index_heap.cuh:58-176)
 * ------------------------------------------------------------------------------------------- */

float gdo_dist2(const float *a, const float *b) {
    float dx = a[0] - b[0];
    float dy = a[1] - b[1];
    float dz = a[2] - b[2];
    return fmaf(dz, dz, fmaf(dx, dx, dy * dy));
}

static float box_dist2(const float *qp, const float *lo, const float *hi) {
    float d[3];
    for (int k = 0; k < 3; ++k) {
        float a = lo[k] - qp[k];
        float b = qp[k] - hi[k];
        float m = a > 0.f ? a : 0.f;
        d[k] = m > b ? m : b;
    }
    return fmaf(d[2], d[2], fmaf(d[0], d[0], d[1] * d[1]));
}

static uint64_t make_key(float d2, uint32_t code) {
    uint32_t bits;
    memcpy(&bits, &d2, 4);
    return ((uint64_t)bits << 32) | code;
}

static float key_d2(uint64_t k) {
    uint32_t bits = (uint32_t)(k >> 32);
    float f;
    memcpy(&f, &bits, 4);
    return f;
}

/* replace the heap maximum by cand and sift down (index_heap.cuh:148-174) */
static void heap_replace_top(uint64_t *h, int K, uint64_t cand) {
    int slot = 0;
    for (;;) {
        int child = 2 * slot + 1;
        if (child >= K) break;
        uint64_t cv = h[child];
        if (child + 1 < K && h[child + 1] > cv) {
            cv = h[child + 1];
            ++child;
        }
        if (cv < cand) break;
        h[slot] = cv;
        slot = child;
    }
    h[slot] = cand;
}

static int cmp_u64(const void *a, const void *b) {
    uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
    return (x > y) - (x < y);
}

static void heap_init(uint64_t *h, int K, float qr) {
    uint64_t sentinel = make_key(qr * qr, 0xffffffffu);
    for (int s = 0; s < K; ++s) h[s] = sentinel;
}

static void write_row(const uint64_t *h, int K, int32_t *codes, float *d2) {
    for (int s = 0; s < K; ++s) {
        uint32_t c = (uint32_t)h[s];
        codes[s] = (c == 0xffffffffu) ? -1 : (int32_t)c;
        if (d2) d2[s] = (c == 0xffffffffu) ? 0.f : key_d2(h[s]);
    }
}

static void empty_row(int K, int32_t *codes, float *d2) {
    for (int s = 0; s < K; ++s) {
        codes[s] = -1;
        if (d2) d2[s] = 0.f;
    }
}

static uint32_t site_code(const float *s4) {
    uint32_t c;
    memcpy(&c, &s4[3], 4);
    return c;
}

void gdo_knn_brute(int n, const float *site4, const float *q, const unsigned char *active, int K, int32_t *codes,
                   float *d2, int threads) {
#pragma omp parallel num_threads(threads > 0 ? threads : 1)
    {
        uint64_t *h = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)K);
#pragma omp for schedule(dynamic, 16)
        for (int i = 0; i < n; ++i) {
            int32_t *crow = codes + (size_t)i * K;
            float *drow = d2 ? d2 + (size_t)i * K : NULL;
            if (!active[i]) {
                empty_row(K, crow, drow);
                continue;
            }
            heap_init(h, K, q[i]);
            float cut = key_d2(h[0]);
            const float *qp = site4 + 4 * (size_t)i;
            for (int j = 0; j < n; ++j) {
                if (!active[j]) continue;
                float dd = gdo_dist2(qp, site4 + 4 * (size_t)j);
                if (!(dd <= cut)) continue;
                uint64_t cand = make_key(dd, site_code(site4 + 4 * (size_t)j));
                if (cand < h[0]) {
                    heap_replace_top(h, K, cand);
                    cut = key_d2(h[0]);
                }
            }
            qsort(h, (size_t)K, sizeof(uint64_t), cmp_u64);
            write_row(h, K, crow, drow);
        }
        free(h);
    }
}

/* replace slot `slot` by the smaller cand and sift it down (index_heap.cuh:133-174) */
static void heap_replace_at(uint64_t *h, int K, int slot, uint64_t cand) {
    for (;;) {
        int child = 2 * slot + 1;
        if (child >= K) break;
        uint64_t cv = h[child];
        if (child + 1 < K && h[child + 1] > cv) {
            cv = h[child + 1];
            ++child;
        }
        if (cv < cand) break;
        h[slot] = cv;
        slot = child;
    }
    h[slot] = cand;
}

/* The Morton ghost rule (morton_gcount, inc/swarm/morton/morton_ghost.cuh:28-50): particle i's
 * image 2 (+width) is kept when its seam distance to the x_min plane is at most q_max, image 1
 * (-width) when its distance to the x_max plane is.  `point` holds the physical float sites (x, y, z,
 * code) and `posx` the float azimuths; keep[2i] is image 1, keep[2i+1] image 2.  The seam distance
 * is computed in double from the float inputs and `margin` is returned for each decision as
 * (distance - q_max) / q_max, so a checker can set aside decisions closer than float rounding. */
void gdo_morton_ghosts(int n, const float *site4, const float *posx, float q_max, float x_min, float x_max,
                       unsigned char *keep, double *margin) {
    for (int i = 0; i < n; ++i) {
        const double R = hypot((double)site4[4 * (size_t)i], (double)site4[4 * (size_t)i + 1]);
        const float off[2] = {x_max - posx[i], posx[i] - x_min};
        for (int image = 0; image < 2; ++image) {
            const double c = cos((double)off[image]);
            const double d = (c >= 0.0) ? R * fabs(sin((double)off[image])) : R;
            keep[2 * (size_t)i + image] = d <= (double)q_max;
            margin[2 * (size_t)i + image] = q_max > 0.f ? (d - q_max) / q_max : d;
        }
    }
}

void gdo_knn_brute_images(int n, int n_sites, const float *site4, const float *q, const unsigned char *active,
                          int K, float image_dist_min, float q_dedup, int32_t *codes, float *d2, int threads) {
#pragma omp parallel num_threads(threads > 0 ? threads : 1)
    {
        uint64_t *h = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)K);
#pragma omp for schedule(dynamic, 16)
        for (int i = 0; i < n; ++i) {
            int32_t *crow = codes + (size_t)i * K;
            float *drow = d2 ? d2 + (size_t)i * K : NULL;
            if (!active[i]) {
                empty_row(K, crow, drow);
                continue;
            }
            /* unique_ids (_col_cache.cuh:38-39; swarm_runtime.cu:413-415 with q_dedup = max q) */
            const float qd = q_dedup >= 0.f ? q_dedup : q[i];
            const int dedup = !(image_dist_min < 0.f || image_dist_min > 2.0f * qd);
            heap_init(h, K, q[i]);
            const float *qp = site4 + 4 * (size_t)i;
            for (int j = 0; j < n_sites; ++j) {
                const uint32_t code = site_code(site4 + 4 * (size_t)j);
                if (code == 0xffffffffu) continue; /* an image the Morton ghost rule dropped */
                const uint32_t idx_old = code / 3u;
                if (!active[idx_old]) continue;
                const uint64_t cand = make_key(gdo_dist2(qp, site4 + 4 * (size_t)j), code);
                /* processCandidate (index_heap.cuh:112-176) */
                int slot = -1;
                if (dedup)
                    for (int s = 0; s < K; ++s) {
                        const uint32_t old = (uint32_t)h[s];
                        if (old == 0xffffffffu || old / 3u != idx_old) continue;
                        slot = s;
                        break;
                    }
                if (slot >= 0) {
                    if (cand >= h[slot]) continue;
                } else {
                    if (cand >= h[0]) continue;
                    slot = 0;
                }
                heap_replace_at(h, K, slot, cand);
            }
            qsort(h, (size_t)K, sizeof(uint64_t), cmp_u64);
            write_row(h, K, crow, drow);
        }
        free(h);
    }
}

/* ---- KD tree: widest-dimension median splits over active sites ----------------------------- */
typedef struct {
    float lo[3], hi[3];
    int begin, end;   /* range in the permuted index array */
    int left, right;  /* children, -1 for a leaf */
} onode;

typedef struct {
    onode *node;
    int count, cap;
    int *idx;
    const float *site4;
} otree;

#define OLEAF 8

static int tree_push(otree *t) {
    if (t->count == t->cap) {
        t->cap = t->cap ? 2 * t->cap : 1024;
        t->node = (onode *)realloc(t->node, sizeof(onode) * (size_t)t->cap);
    }
    return t->count++;
}

static float coord(const otree *t, int id, int dim) { return t->site4[4 * (size_t)id + dim]; }

/* quickselect: put the element of rank k (by coordinate dim, ties by index) at position k */
static void select_k(otree *t, int lo, int hi, int k, int dim) {
    int *a = t->idx;
    while (hi - lo > 1) {
        int mid = lo + (hi - lo) / 2;
        int piv = a[mid];
        float pv = coord(t, piv, dim);
        int i = lo, j = hi - 1;
        a[mid] = a[j];
        a[j] = piv;
        int store = lo;
        for (i = lo; i < j; ++i) {
            float v = coord(t, a[i], dim);
            if (v < pv || (v == pv && a[i] < piv)) {
                int tmp = a[i];
                a[i] = a[store];
                a[store] = tmp;
                ++store;
            }
        }
        a[j] = a[store];
        a[store] = piv;
        if (store == k) return;
        if (k < store) hi = store;
        else lo = store + 1;
    }
}

static int tree_build(otree *t, int begin, int end) {
    int id = tree_push(t);
    onode nd;
    for (int k = 0; k < 3; ++k) {
        nd.lo[k] = INFINITY;
        nd.hi[k] = -INFINITY;
    }
    for (int i = begin; i < end; ++i)
        for (int k = 0; k < 3; ++k) {
            float v = coord(t, t->idx[i], k);
            if (v < nd.lo[k]) nd.lo[k] = v;
            if (v > nd.hi[k]) nd.hi[k] = v;
        }
    nd.begin = begin;
    nd.end = end;
    nd.left = nd.right = -1;
    if (end - begin > OLEAF) {
        int dim = 0;
        float w = nd.hi[0] - nd.lo[0];
        for (int k = 1; k < 3; ++k)
            if (nd.hi[k] - nd.lo[k] > w) {
                w = nd.hi[k] - nd.lo[k];
                dim = k;
            }
        int mid = begin + (end - begin) / 2;
        select_k(t, begin, end, mid, dim);
        int l = tree_build(t, begin, mid);
        int r = tree_build(t, mid, end);
        nd.left = l;
        nd.right = r;
    }
    t->node[id] = nd;
    return id;
}

void *gdo_kdtree_build(int n, const float *site4, const unsigned char *active) {
    otree *t = (otree *)calloc(1, sizeof(otree));
    t->site4 = site4;
    t->idx = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    int m = 0;
    for (int i = 0; i < n; ++i)
        if (active[i]) t->idx[m++] = i;
    if (m > 0) tree_build(t, 0, m);
    return t;
}

void gdo_kdtree_free(void *tp) {
    otree *t = (otree *)tp;
    if (!t) return;
    free(t->node);
    free(t->idx);
    free(t);
}

void gdo_kdtree_query(void *tp, int n, const float *q, const unsigned char *active, int K, int32_t *codes, float *d2,
                      int threads, int first, int count) {
    otree *t = (otree *)tp;
    const float *site4 = t->site4;
    if (count < 0) count = n - first;
#pragma omp parallel num_threads(threads > 0 ? threads : 1)
    {
        uint64_t *h = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)K);
        int stack[128];
#pragma omp for schedule(dynamic, 64)
        for (int i = first; i < first + count; ++i) {
            int32_t *crow = codes + (size_t)i * K;
            float *drow = d2 ? d2 + (size_t)i * K : NULL;
            if (!active[i] || t->count == 0) {
                empty_row(K, crow, drow);
                continue;
            }
            heap_init(h, K, q[i]);
            float cut = key_d2(h[0]);
            const float *qp = site4 + 4 * (size_t)i;
            int sp = 0;
            stack[sp++] = 0;
            while (sp > 0) {
                const onode *nd = &t->node[stack[--sp]];
                if (!(box_dist2(qp, nd->lo, nd->hi) <= cut)) continue;
                if (nd->left < 0) {
                    for (int k = nd->begin; k < nd->end; ++k) {
                        int j = t->idx[k];
                        float dd = gdo_dist2(qp, site4 + 4 * (size_t)j);
                        if (!(dd <= cut)) continue;
                        uint64_t cand = make_key(dd, site_code(site4 + 4 * (size_t)j));
                        if (cand < h[0]) {
                            heap_replace_top(h, K, cand);
                            cut = key_d2(h[0]);
                        }
                    }
                    continue;
                }
                const onode *l = &t->node[nd->left], *r = &t->node[nd->right];
                float dl = box_dist2(qp, l->lo, l->hi), dr = box_dist2(qp, r->lo, r->hi);
                if (dl <= dr) {
                    stack[sp++] = nd->right;
                    stack[sp++] = nd->left;
                } else {
                    stack[sp++] = nd->left;
                    stack[sp++] = nd->right;
                }
            }
            qsort(h, (size_t)K, sizeof(uint64_t), cmp_u64);
            write_row(h, K, crow, drow);
        }
        free(h);
    }
}

void gdo_knn_kdtree(int n, const float *site4, const float *q, const unsigned char *active, int K, int32_t *codes,
                    float *d2, int threads, int first, int count) {
    void *t = gdo_kdtree_build(n, site4, active);
    gdo_kdtree_query(t, n, q, active, K, codes, d2, threads, first, count);
    gdo_kdtree_free(t);
}

/* ---------------------------------------------------------------------------------------------
 * _get_ball_measure (inc/swarm/_collision.cuh:66-115)
 * ------------------------------------------------------------------------------------------- */
static double ball_measure(const gd_config *c, double y, double z, double radius) {
    if (radius <= 0.0) return 0.0;
    if (c->n_x == 1 && c->n_z == 1) {
        double R_lo = fmax(c->y_min, y - radius);
        double R_hi = fmin(c->y_max, y + radius);
        return (R_hi > R_lo) ? M_PI * (R_hi * R_hi - R_lo * R_lo) : 0.0;
    }
    int dim = 1 + (c->n_x > 1) + (c->n_z > 1);
    double measure = (dim == 1) ? 2.0 * radius
                     : (dim == 2) ? M_PI * radius * radius
                                  : 4.0 * M_PI * radius * radius * radius / 3.0;
    double distances[4] = {y - c->y_min, c->y_max - y, 1.0e+100, 1.0e+100};
    if (c->n_z > 1) {
        distances[2] = y * (z - c->z_min);
        distances[3] = y * (c->z_max - z);
    }
    int bounds = (c->n_z > 1) ? 4 : 2;
    for (int b = 0; b < bounds; ++b) {
        double d = fmax(0.0, distances[b]);
        if (d >= radius) continue;
        if (dim == 1) {
            measure *= 0.5 * (1.0 + d / radius);
        } else if (dim == 2) {
            double cap = radius * radius * acos(d / radius) - d * sqrt(radius * radius - d * d);
            measure *= 1.0 - cap / (M_PI * radius * radius);
        } else {
            double cap = M_PI * (radius - d) * (radius - d) * (2.0 * radius + d) / 3.0;
            measure *= 1.0 - cap / (4.0 * M_PI * radius * radius * radius / 3.0);
        }
    }
    if (c->n_x == 1) measure *= 2.0 * M_PI * cyl_R(c, y, z);
    return measure;
}

void gdo_ball_measure(const gd_config *c, const gd_particle *p, int n, const unsigned char *active, const float *kth,
                      double *measure) {
    for (int i = 0; i < n; ++i)
        measure[i] = active[i] ? ball_measure(c, p[i].position[1], p[i].position[2], sqrt((double)kth[i])) : 0.0;
}

/* col_space_bin (src/swarm/col_space_bin.cu:11-35) */
void gdo_space_bin(const gd_config *c, const gd_particle *p, int n, int32_t *spatial) {
    for (int i = 0; i < n; ++i) {
        double x = p[i].position[0], y = p[i].position[1], z = p[i].position[2];
        int bx = 0, bz = 0;
        int by = (int)floor((y - c->y_min) / (c->y_max - c->y_min) * c->col_bin_y);
        if (c->n_x > 1) bx = (int)floor((x - c->x_min) / (c->x_max - c->x_min) * c->col_bin_x);
        if (c->n_z > 1) bz = (int)floor((z - c->z_min) / (c->z_max - c->z_min) * c->col_bin_z);
        bx = bx < 0 ? 0 : (bx >= c->col_bin_x ? c->col_bin_x - 1 : bx);
        by = by < 0 ? 0 : (by >= c->col_bin_y ? c->col_bin_y - 1 : by);
        bz = bz < 0 ? 0 : (bz >= c->col_bin_z ? c->col_bin_z - 1 : bz);
        int cx = (c->n_x > 1) ? c->col_bin_x : 1;
        spatial[i] = bx + cx * (by + c->col_bin_y * bz);
    }
}
