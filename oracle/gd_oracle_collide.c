/*
 * gd_oracle_collide.c -- CPU restatement of the frozen-bath collision operator's per-owner
 * arithmetic (test infrastructure only; see gd_oracle.h).
 *
 *   gdo_env               _cache_query_environment   inc/swarm/_col_rates.cuh:13-24
 *   gdo_pair_speed_cached _cached_pair_velocity      inc/swarm/_col_rates.cuh:127-141
 *   gdo_pair_speed_direct _get_vrel_pair (analytic)  inc/swarm/_collision.cuh:277-325
 *   gdo_outcome_moments   _erosion_outcome_moments   inc/swarm/_col_event.cuh:258-301
 *   gdo_sample_outcome    _sample_erosion_outcome    inc/swarm/_col_event.cuh:306-336
 *   gdo_bath_rate         col_bath_rate              src/swarm/col_bath_rate.cu:13-130
 *   gdo_chain_owner       col_skip_scan + col_chain_run for one owner and one bath
 *                         src/swarm/col_skip_scan.cu:13-59, src/swarm/col_chain_run.cu:21-404
 *
 * The chain takes its uniform deviates from an array (the values _get_col_uniform draws from the
 * owner's XORWOW stream), so the oracle replays exactly the device's random sequence without
 * re-implementing the generator.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "gd_oracle.h"

static double cyl_R(const gd_config *c, double y, double z) { return (c->n_z > 1) ? y * sin(z) : y; }
static double cyl_Z(const gd_config *c, double y, double z) { return (c->n_z > 1) ? y * cos(z) : 0.0; }
static double get_hg(const gd_config *c, double R) { return c->aspr_0 * pow(R / c->R_0, 0.5 * (c->idx_q + 1.0)); }
static double grain_mass(const gd_config *c, double s) { return M_PI * c->rho_0 * s * s * s / 6.0; }
static double omega_k(const gd_config *c, double R) { return sqrt(c->G * c->M_S / R / R / R); }
static double get_eta(const gd_config *c, double R, double Z, double h) {
    return -0.5 * ((c->idx_p + 0.5 * c->idx_q - 1.5) * h * h + c->idx_q * (1.0 - R / sqrt(R * R + Z * Z)));
}
static double gas_strat(double R, double Z, double h) { return exp((R / sqrt(R * R + Z * Z) - 1.0) / (h * h)); }
static double sigma_g(const gd_config *c, double R) { return c->sigma_0 * pow(R / c->R_0, c->idx_p); }
static double sound_speed(const gd_config *c, double R, double h) { return h * omega_k(c, R) * R; }
static double get_alpha(const gd_config *c, double R, double h) {
    if (c->const_nu) return c->nu / (h * h * R * R * omega_k(c, R));
    return c->alpha;
}
static double re_inv_sqrt(const gd_config *c, double R, double alpha, double sig) {
    double re;
    if (c->code_unit) {
        double alpha_0 = get_alpha(c, c->R_0, c->aspr_0);
        re = c->reynolds_0 * (alpha / alpha_0) * (sig / c->sigma_0);
    } else {
        re = 0.5 * alpha * sig * c->x_sec / c->m_mol;
    }
    return 1.0 / sqrt(re);
}

/* the six Ormel-Cuzzi regimes (_collision.cuh:153-273 / _col_rates.cuh:34-124) */
static double oc07(double st_i, double st_j, double re_inv, double vg_sq) {
    double sl = st_i >= st_j ? st_i : st_j;
    double ss = st_i >= st_j ? st_j : st_i;
    double eps = ss / sl;
    double y_a = 1.6, y_s = 1.6015125;
    y_s += -0.63119577 * sl;
    y_s += 0.32938936 * sl * sl;
    y_s += -0.29847604 * sl * sl * sl;
    double v2;
    if (sl < 0.2 * re_inv) {
        v2 = vg_sq * (sl - ss) * (sl - ss) / re_inv;
    } else if (sl < re_inv / y_a) {
        v2 = vg_sq * (sl - ss) / (sl + ss);
        v2 *= (sl / (1.0 + re_inv / sl) - ss / (1.0 + re_inv / ss));
    } else if (sl < 5.0 * re_inv) {
        double c = (sl - ss) / (sl + ss);
        c *= (sl / (1.0 + y_a) - ss * ss / (ss + y_a * sl));
        c += 2.0 * (y_a * sl - re_inv) + sl / (1.0 + y_a);
        c -= sl * sl / (sl + re_inv);
        c += ss * ss / (y_a * sl + ss);
        c -= ss * ss / (ss + re_inv);
        v2 = vg_sq * c;
    } else if (sl < 0.2) {
        v2 = vg_sq * sl;
        v2 *= (2.0 * y_a - (1.0 + eps) + 2.0 / (1.0 + eps) * (1.0 / (1.0 + y_a) + eps * eps * eps / (y_a + eps)));
    } else if (sl < 1.0) {
        v2 = vg_sq * sl;
        v2 *= (2.0 * y_s - (1.0 + eps) + 2.0 / (1.0 + eps) * (1.0 / (1.0 + y_s) + eps * eps * eps / (y_s + eps)));
    } else {
        v2 = vg_sq * (1.0 / (1.0 + sl) + 1.0 / (1.0 + ss));
    }
    return sqrt(v2);
}

/* env = {Z, omega, vn, radial, strat, cs, re_inv_sqrt, vg_sq} */
void gdo_env(const gd_config *c, double y, double z, double *env) {
    double R = cyl_R(c, y, z), Z = cyl_Z(c, y, z);
    double h = get_hg(c, R);
    double omega = omega_k(c, R);
    double cs = sound_speed(c, R, h);
    double alpha = get_alpha(c, R, h);
    double strat = gas_strat(R, Z, h);
    env[0] = Z;
    env[1] = omega;
    env[2] = -get_eta(c, R, Z, h) * R * omega;
    env[3] = pow(R / c->R_0, c->idx_p);
    env[4] = strat;
    env[5] = cs;
    env[6] = re_inv_sqrt(c, R, alpha, sigma_g(c, R) * strat);
    env[7] = 1.5 * alpha * cs * cs;
}

double gdo_pair_speed_cached(const gd_config *c, const double *e, double size_i, double size_j) {
    double si = c->stokes_0 * (size_i / c->S_0);
    si /= e[3];
    si /= e[4];
    double sj = c->stokes_0 * (size_j / c->S_0);
    sj /= e[3];
    sj /= e[4];
    double fi = 1.0 / (1.0 + si * si);
    double fj = 1.0 / (1.0 + sj * sj);
    double dvr = 2.0 * e[2] * fma(si, fi, -(sj * fj));  /* the device's pinned contraction */
    double dvphi = e[2] * (fi - fj);
    double dvz = e[0] * e[1] * (fmin(si, 0.5) - fmin(sj, 0.5));
    double vt = oc07(si, sj, e[6], e[7]);
    double mi = grain_mass(c, size_i), mj = grain_mass(c, size_j);
    double vb = fmin(sqrt(8.0 * e[5] * e[5] * c->m_mol * (mi + mj) / (M_PI * mi * mj)), e[5]);
    return sqrt(dvr * dvr + dvphi * dvphi + dvz * dvz + vt * vt + vb * vb);
}

static double stokes_at(const gd_config *c, double R, double Z, double h, double size) {
    double st = c->stokes_0 * (size / c->S_0);
    if (!c->const_st) {
        st /= pow(R / c->R_0, c->idx_p);
        st /= gas_strat(R, Z, h);
    }
    return st;
}

double gdo_pair_speed_direct(const gd_config *c, double y, double z, double size_i, double size_j) {
    double R = cyl_R(c, y, z), Z = cyl_Z(c, y, z);
    double h = get_hg(c, R);
    double omega = omega_k(c, R);
    double si = stokes_at(c, R, Z, h, size_i);
    double sj = stokes_at(c, R, Z, h, size_j);
    double vn = -get_eta(c, R, Z, h) * R * omega;
    double fi = 1.0 / (1.0 + si * si);
    double fj = 1.0 / (1.0 + sj * sj);
    double dvr = 2.0 * vn * fma(si, fi, -(sj * fj));  /* the device's pinned contraction */
    double dvphi = vn * (fi - fj);
    double dvz = Z * omega * (fmin(si, 0.5) - fmin(sj, 0.5));
    double sigma_local = sigma_g(c, R) * gas_strat(R, Z, h);
    double cs = sound_speed(c, R, h);
    double alpha = get_alpha(c, R, h);
    double vt = oc07(si, sj, re_inv_sqrt(c, R, alpha, sigma_local), 1.5 * alpha * cs * cs);
    double vb = 0.0;
    if (!c->code_unit) {
        double mi = grain_mass(c, size_i), mj = grain_mass(c, size_j);
        double v = sqrt(8.0 * cs * cs * c->m_mol * (mi + mj) / (M_PI * mi * mj));
        vb = fmin(v, cs);
    }
    return sqrt(dvr * dvr + dvphi * dvphi + dvz * dvz + vt * vt + vb * vb);
}

static double sticking_packet(double q) { return q > 0.0 && q <= 1.0e-06 ? fmax(1.0, floor(1.0e-04 / q)) : 1.0; }
static double mass_ratio(double si, double sj) {
    double r = sj / si;
    return r * r * r;
}

/* out = {mean, second, maximum}; returns the channel factor */
double gdo_outcome_moments(const gd_config *c, double si, double sj, int high, double *out) {
    double q = mass_ratio(si, sj);
    double G = sticking_packet(q);
    if (!high) {
        double mean = log1p(G * q) / 3.0;
        out[0] = mean;
        out[1] = mean * mean;
        out[2] = mean;
        return 1.0 / G;
    }
    if (q <= 0.1) {
        double remnant = (1.0 - q) / G, debris = q, factor = remnant + debris;
        double jr = -log1p(-G * q) / 3.0;
        double jd = -log(q) / 3.0;
        out[0] = (remnant * jr + debris * jd) / factor;
        out[1] = (remnant * jr * jr + debris * jd * jd) / factor;
        out[2] = fmax(jr, jd);
        return factor;
    }
    double L = 0.5 * log(si / c->init_smin);
    if (L < 1.0e-03) {
        out[0] = L - L * L / 6.0 + L * L * L * L / 360.0;
        out[1] = L * L * (4.0 / 3.0 - L / 3.0 + L * L / 90.0 + L * L * L / 180.0);
    } else {
        double tail = exp(-L) / (-expm1(-L));
        out[0] = 2.0 * (1.0 - L * tail);
        out[1] = 8.0 - (4.0 * L * L + 8.0 * L) * tail;
    }
    out[2] = 2.0 * L;
    return 1.0;
}

double gdo_sample_outcome(const gd_config *c, double si, double sj, int high, double u) {
    double q = mass_ratio(si, sj);
    double G = sticking_packet(q);
    if (!high) return cbrt(si * si * si + G * sj * sj * sj);
    if (q <= 0.1) {
        double factor = (1.0 - q) / G + q;
        if (u < q / factor) return sj;
        return si * cbrt(1.0 - G * q);
    }
    double lower = sqrt(c->init_smin);
    double root = lower + u * (sqrt(si) - lower);
    return fmin(si, fmax(c->init_smin, root * root));
}

/* one owner's per-slot pair rate (_get_col_chain_rate / measure), vrel out */
static double pair_rate(const gd_config *c, const gd_particle *p, int i, int j, double size_i, double size_j,
                        double numr_j, double measure, double lambda0, const double *env, double *vrel) {
    double r;
    *vrel = 0.0;
    if (c->coag_kernel == 0) {
        r = lambda0 * numr_j;
    } else if (c->coag_kernel == 1) {
        r = lambda0 * numr_j * (grain_mass(c, size_i) + grain_mass(c, size_j));
    } else if (c->coag_kernel == 2) {
        r = lambda0 * numr_j * grain_mass(c, size_i) * grain_mass(c, size_j);
    } else {
        double y = p[i].position[1], z = p[i].position[2];
        *vrel = (!c->code_unit && !c->const_st) ? gdo_pair_speed_cached(c, env, size_i, size_j)
                                                : gdo_pair_speed_direct(c, y, z, size_i, size_j);
        r = numr_j * *vrel * M_PI * (size_i + size_j) * (size_i + size_j) / 4.0;
        if (c->n_z == 1) {
            double Ri = cyl_R(c, y, z);
            double Rj = cyl_R(c, p[j].position[1], p[j].position[2]);
            double Hi = Ri * get_hg(c, Ri), Hj = Rj * get_hg(c, Rj);
            r /= sqrt(2.0 * M_PI * (Hi * Hi + Hj * Hj));
        }
    }
    return r / measure;
}

/* one pair between owner (yi, zi) and partner (yj, zj), as col_bath_rate evaluates it */
double gdo_pair_rate(const gd_config *c, double yi, double zi, double yj, double zj, double size_i, double size_j,
                     double numr_j, double lambda0, double measure, double *vrel) {
    gd_particle p[2];
    memset(p, 0, sizeof(p));
    p[0].position[1] = yi;
    p[0].position[2] = zi;
    p[1].position[1] = yj;
    p[1].position[2] = zj;
    double env[8] = {0};
    if (c->coag_kernel == 3 && yi > 0.0) gdo_env(c, yi, zi, env);
    return pair_rate(c, p, 0, 1, size_i, size_j, numr_j, measure, lambda0, env, vrel);
}

/* slot arrays for one owner; returns nothing, fills rate/j1/j2/jm/last */
static void owner_slots(const gd_config *c, const gd_particle *p, int i, const int32_t *row, double size_i,
                        const double *size_old, const double *numr_old, double measure, double lambda0,
                        const double *env, double *rate, double *j1, double *j2, double *jm) {
    int K = c->n_k;
    for (int s = 0; s < K; ++s) {
        rate[s] = j1[s] = j2[s] = jm[s] = 0.0;
        int nb = row[s];
        if (nb < 0) continue;
        int j = nb / 3;
        double vrel;
        double pr = pair_rate(c, p, i, j, size_i, size_old[j], numr_old[j], measure, lambda0, env, &vrel);
        double mom[3] = {0, 0, 0};
        pr *= gdo_outcome_moments(c, size_i, size_old[j], vrel >= c->v_frag, mom);
        rate[s] = pr;
        j1[s] = pr * mom[0];
        j2[s] = pr * mom[1];
        jm[s] = pr > 0.0 ? mom[2] : 0.0;
    }
}

/* the (count+1)/2 fold of col_bath_rate.cu:105-118 and col_chain_run.cu:230-245 */
static void fold(int K, double *a, double *b, double *c2, double *mx, int *ok, int *last) {
    for (int count = K; count > 1; count = (count + 1) / 2) {
        int half = (count + 1) / 2;
        for (int j = 0; j < count / 2; ++j) {
            a[j] += a[j + half];
            b[j] += b[j + half];
            c2[j] += c2[j + half];
            mx[j] = fmax(mx[j], mx[j + half]);
            if (ok) ok[j] = ok[j] && ok[j + half];
            if (last) {
                int l = last[j], r = last[j + half];
                last[j] = (l == -2 || r == -2) ? -2 : (l > r ? l : r);
            }
        }
    }
}

void gdo_bath_rate(const gd_config *c, int n, const gd_particle *p, const int32_t *codes, const double *measure,
                   const unsigned char *active, const double *size_old, const double *numr_old, double lambda0,
                   double *cached, double *rate_out, double *change_out, double *second_out, int threads) {
    int K = c->n_k;
#pragma omp parallel num_threads(threads > 0 ? threads : 1)
    {
        double *w = (double *)malloc(sizeof(double) * 4 * (size_t)K);
        int *ok = (int *)malloc(sizeof(int) * (size_t)K);
#pragma omp for schedule(dynamic, 64)
        for (int i = 0; i < n; ++i) {
            double *r = w, *a = w + K, *b = w + 2 * K, *m = w + 3 * K;
            double env[8] = {0};
            if (c->coag_kernel == 3 && p[i].position[1] > 0.0) gdo_env(c, p[i].position[1], p[i].position[2], env);
            for (int s = 0; s < K; ++s) r[s] = a[s] = b[s] = m[s] = 0.0;
            if (active[i] && measure[i] > 0.0)
                owner_slots(c, p, i, codes + (size_t)i * K, size_old[i], size_old, numr_old, measure[i], lambda0, env,
                            r, a, b, m);
            for (int s = 0; s < K; ++s) ok[s] = isfinite(r[s]) && r[s] >= 0.0;
            fold(K, r, a, b, m, ok, NULL);
            cached[4 * (size_t)i + 0] = ok[0] ? r[0] : -1.0;
            cached[4 * (size_t)i + 1] = a[0];
            cached[4 * (size_t)i + 2] = b[0];
            cached[4 * (size_t)i + 3] = m[0];
            rate_out[i] = r[0];
            change_out[i] = a[0];
            second_out[i] = b[0];
        }
        free(w);
        free(ok);
    }
}

static double col_uniform(const double *u, int nu, int *used, int *overrun) {
    if (*used >= nu) {
        *overrun = 1;
        return 0.5;
    }
    return u[(*used)++];
}

/*
 * One owner through skip-scan + chain for one bath that starts at time 0 with zero compensators.
 * state in/out: [0] size, [1] numr; out: [2] time, [3] hazard, [4] jump1, [5] jump2, [6] jumpmax,
 * [7] events.  Returns the chain error code (0..6), or 8 if the uniform array ran out.
 * *used receives the number of deviates consumed (committed) from u.
 */
int gdo_chain_owner(const gd_config *c, int i, const gd_particle *p, const int32_t *codes, const double *measure,
                    const unsigned char *active, const double *size_old, const double *numr_old, double lambda0,
                    double bath_end, const double *cached4, const double *u, int nu, double *state, int *used) {
    int K = c->n_k;
    double size_i = state[0], numr_i = state[1];
    double time_i = 0.0, hazard = 0.0, jump1 = 0.0, jump2 = 0.0, jumpmax = 0.0;
    int events = 0, err = 0, overrun = 0;
    *used = 0;
    if (!active[i] || !(measure[i] > 0.0)) {
        time_i = bath_end;
        goto done;
    }
    /* col_skip_scan: cached first waiting time */
    {
        double rate = cached4[0];
        if (isfinite(rate) && rate >= 0.0) {
            if (rate == 0.0) {
                time_i = bath_end;
                goto done;
            }
            double U = fmin(u[0], nextafter(1.0, 0.0));
            double wait = -log(U) / rate;
            double remaining = bath_end - time_i;
            if (isfinite(wait) && wait > 0.0 && wait >= remaining) {
                hazard += rate * remaining;
                jump1 += cached4[1] * remaining;
                jump2 += cached4[2] * remaining;
                jumpmax = fmax(jumpmax, cached4[3]);
                time_i = bath_end;
                *used = 1;
                goto done;
            }
        }
    }
    {
        double env[8] = {0};
        if (c->coag_kernel == 3 && p[i].position[1] > 0.0) gdo_env(c, p[i].position[1], p[i].position[2], env);
        double *w = (double *)malloc(sizeof(double) * 5 * (size_t)K);
        int *last = (int *)malloc(sizeof(int) * (size_t)K);
        double *prate = w, *tot = w + K, *j1 = w + 2 * K, *j2 = w + 3 * K, *jm = w + 4 * K;
        const int32_t *row = codes + (size_t)i * K;
        for (;;) {
            owner_slots(c, p, i, row, size_i, size_old, numr_old, measure[i], lambda0, env, prate, j1, j2, jm);
            for (int s = 0; s < K; ++s) {
                tot[s] = prate[s];
                last[s] = (!isfinite(prate[s]) || prate[s] < 0.0) ? -2 : (prate[s] > 0.0 ? s : -1);
            }
            fold(K, tot, j1, j2, jm, NULL, last);
            double total = tot[0];
            if (last[0] == -2) { err = 1; break; }
            if (!isfinite(total) || total < 0.0) { err = 2; break; }
            if (total == 0.0) { time_i = bath_end; break; }
            double U = fmin(col_uniform(u, nu, used, &overrun), nextafter(1.0, 0.0));
            double wait = -log(U) / total;
            double remaining = bath_end - time_i;
            if (!isfinite(wait) || !(wait > 0.0)) { err = 3; break; }
            if (wait >= remaining) {
                hazard += total * remaining;
                jump1 += j1[0] * remaining;
                jump2 += j2[0] * remaining;
                jumpmax = fmax(jumpmax, jm[0]);
                time_i = bath_end;
                break;
            }
            double event_time = time_i + wait;
            if (!(event_time > time_i)) { err = 4; break; }
            hazard += total * wait;
            jump1 += j1[0] * wait;
            jump2 += j2[0] * wait;
            jumpmax = fmax(jumpmax, jm[0]);
            double target = fmin(col_uniform(u, nu, used, &overrun), nextafter(1.0, 0.0)) * total;
            double cum = 0.0;
            int pick = -1;
            for (int s = 0; s < K; ++s) {
                if (prate[s] <= 0.0) continue;
                cum += prate[s];
                if (cum > target) { pick = s; break; }
            }
            if (pick < 0) pick = last[0];
            if (pick < 0) { err = 5; break; }
            int j = row[pick] / 3;
            double size_j = size_old[j];
            double vrel = 0.0;
            if (c->coag_kernel == 3)
                vrel = (!c->code_unit && !c->const_st) ? gdo_pair_speed_cached(c, env, size_i, size_j)
                                                       : gdo_pair_speed_direct(c, p[i].position[1], p[i].position[2],
                                                                               size_i, size_j);
            double mass_before = numr_i * size_i * size_i * size_i;
            int high = vrel >= c->v_frag;
            double sample = high ? fmin(col_uniform(u, nu, used, &overrun), nextafter(1.0, 0.0)) : 0.0;
            double size_new = gdo_sample_outcome(c, size_i, size_j, high, sample);
            numr_i = mass_before / (size_new * size_new * size_new);
            size_i = size_new;
            time_i = event_time;
            ++events;
            double mass_after = numr_i * size_i * size_i * size_i;
            double scale = fmax(fabs(mass_before), fabs(mass_after));
            if (!isfinite(size_i) || !isfinite(numr_i) || !(size_i > 0.0) || !(numr_i > 0.0) ||
                fabs(mass_after - mass_before) > 2.0e-12 * scale) { err = 6; break; }
            if (overrun) break;
        }
        free(w);
        free(last);
    }
done:
    state[0] = size_i;
    state[1] = numr_i;
    state[2] = time_i;
    state[3] = hazard;
    state[4] = jump1;
    state[5] = jump2;
    state[6] = jumpmax;
    state[7] = (double)events;
    if (overrun) return 8;
    return err;
}
