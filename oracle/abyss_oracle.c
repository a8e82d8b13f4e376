/* Test infrastructure only: the CPU oracle (checker).  See abyss_oracle.h.
 *
 * Every expression keeps the reference's operation order; the file is
 * compiled with -ffp-contract=off so no multiply-add is fused, which keeps
 * it bit-identical to the reference's own build at eps2 == 0. */
#include "abyss_oracle.h"
#include <math.h>
#include <stdlib.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static void set_threads(int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
}

/* UpdateParticle.cpp:37-59 (the double overload). */
void oracle_predict(int n, const double *x, const double *v, const double *a0,
                    const double *a1, const double *t0, double new_time,
                    double time_scale, double *px, double *pv) {
    for (int j = 0; j < n; ++j) {
        double dt = (new_time - t0[j]) * time_scale;
        for (int d = 0; d < 3; ++d) {
            const int k = 3 * j + d;
            if (dt == 0) {
                px[k] = x[k];
                pv[k] = v[k];
            } else {
                px[k] = ((a1[k] * dt / 3 + a0[k]) * dt / 2 + v[k]) * dt + x[k];
                pv[k] = (a1[k] * dt / 2 + a0[k]) * dt + v[k];
            }
        }
    }
}

/* One target against j in [j0, j1): ComputeAcceleration.cpp:235-299.
 * The reference's "total minus old neighbours" sum (a, adot at :273-282) only
 * feeds its own corrector and is not part of this path's output. */
static int reg_one(int i, int j0, int j1, const double *px, const double *pv,
                   const double *mass, double r2i, double eps2, int cap,
                   double *a_new, double *adot_new, double *a_irr, double *adot_irr,
                   int *list) {
    const double *pi = px + 3 * i, *vi = pv + 3 * i;
    int cnt = 0;
    for (int d = 0; d < 3; ++d) {
        a_new[d] = 0.0;
        adot_new[d] = 0.0;
        if (a_irr) {
            a_irr[d] = 0.0;
            adot_irr[d] = 0.0;
        }
    }
    for (int j = j0; j < j1; ++j) {
        if (j == i) continue;
        double x[3], v[3], r2 = 0.0, vx = 0.0;
        for (int d = 0; d < 3; ++d) {
            x[d] = px[3 * j + d] - pi[d];
            v[d] = pv[3 * j + d] - vi[d];
            r2 += x[d] * x[d];
            vx += v[d] * x[d];
        }
        const double r2s = r2 + eps2;
        const double m_r3 = mass[j] / r2s / sqrt(r2s);
        if (r2 < r2i) {
            if (list && cnt < cap) list[cnt] = j;
            cnt++;
            if (a_irr)
                for (int d = 0; d < 3; ++d) {
                    a_irr[d] += m_r3 * x[d];
                    adot_irr[d] += m_r3 * (v[d] - 3 * x[d] * vx / r2s);
                }
        } else {
            for (int d = 0; d < 3; ++d) {
                a_new[d] += m_r3 * x[d];
                adot_new[d] += m_r3 * (v[d] - 3 * x[d] * vx / r2s);
            }
        }
    }
    return cnt;
}

int oracle_reg_force(int n, const double *px, const double *pv, const double *mass,
                     const double *r2nb, double eps2, int nt, const int *targets,
                     int cap, double *acc_reg, double *jerk_reg, double *acc_irr,
                     double *jerk_irr, int *nnb, int *list, int nthreads) {
    int overflow = 0;
    set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : overflow)
    for (int k = 0; k < nt; ++k) {
        const int i = targets[k];
        const int c = reg_one(i, 0, n, px, pv, mass, r2nb[i], eps2, cap, acc_reg + 3 * k,
                              jerk_reg + 3 * k, acc_irr ? acc_irr + 3 * k : 0,
                              jerk_irr ? jerk_irr + 3 * k : 0,
                              list ? list + (long)k * cap : 0);
        nnb[k] = c;
        if (c > cap) overflow++;
    }
    return overflow;
}

void oracle_reg_force_range(int n, const double *px, const double *pv, const double *mass,
                            const double *r2nb, double eps2, int nt, const int *targets,
                            int j0, int j1, double *acc_reg, double *jerk_reg, int *nnb,
                            int nthreads) {
    (void)n;
    set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1)
    for (int k = 0; k < nt; ++k) {
        const int i = targets[k];
        nnb[k] = reg_one(i, j0, j1, px, pv, mass, r2nb[i], eps2, 0, acc_reg + 3 * k,
                         jerk_reg + 3 * k, 0, 0, 0);
    }
}

/* ComputeAcceleration.cpp:604-636. */
void oracle_hermite_correct(const double *pos, const double *vel, const double *a_reg_old,
                            const double *a_new, const double *adot_new, const double *a_tmp,
                            const double *adot_tmp, double dt, double *new_pos,
                            double *new_vel, double *a2o, double *a3o) {
    const double dt2 = dt * dt;
    const double dt3 = dt2 * dt;
    const double dt4 = dt3 * dt;
    const double dt5 = dt4 * dt;
    for (int d = 0; d < 3; ++d) {
        const double a0 = a_reg_old[2 * d + 0], a1 = a_reg_old[2 * d + 1];
        const double da_dt2 = (a0 - a_new[d] - a_tmp[d]) / dt2;
        const double adot_dt = (a1 + adot_new[d] + adot_tmp[d]) / dt;
        const double a2 = -6 * da_dt2 - 2 * adot_dt - 2 * a1 / dt;
        const double a3 = (12 * da_dt2 + 6 * adot_dt) / dt;
        new_pos[d] = pos[d] + a2 * dt4 / 24 + a3 * dt5 / 120;
        new_vel[d] = vel[d] + a2 * dt3 / 6 + a3 * dt4 / 24;
        a2o[d] = a2;
        a3o[d] = a3;
    }
}

/* TimeStepRoutines.cpp:10-25. */
double oracle_time_step_reg(const double *v, const double *df, double eta) {
    (void)v;
    const double F2 = df[0] * df[0] + df[4] * df[4] + df[8] * df[8];
    const double Fdot2 = df[1] * df[1] + df[5] * df[5] + df[9] * df[9];
    const double F2dot2 = df[2] * df[2] + df[6] * df[6] + df[10] * df[10];
    const double F3dot2 = df[3] * df[3] + df[7] * df[7] + df[11] * df[11];
    double dta = (sqrt(F2 * F2dot2) + Fdot2) / (sqrt(Fdot2 * F3dot2) + F2dot2);
    dta = sqrt(eta * dta);
    return dta;
}

/* TimeStepRoutines.cpp:28-63. */
double oracle_time_step_irr(const double *f, const double *df, double eta) {
    const double F2 = f[0] * f[0] + f[4] * f[4] + f[8] * f[8];
    const double Fdot2 = df[1] * df[1] + df[5] * df[5] + df[9] * df[9];
    const double F2dot2 = df[2] * df[2] + df[6] * df[6] + df[10] * df[10];
    const double F3dot2 = df[3] * df[3] + df[7] * df[7] + df[11] * df[11];
    double ts = (sqrt(F2 * F2dot2) + Fdot2) / (sqrt(Fdot2 * F3dot2) + F2dot2);
    ts = sqrt(eta * ts);
    return ts;
}

/* TimeStepRoutines.cpp:102-115. */
void oracle_block_time_step(double dt, double time_scale, int time_block, int *level,
                            unsigned long long *block, double *step) {
    int lv = (int)floor(log(dt / time_scale) / log(2.0));
    if (lv < time_block) lv = time_block;
    *level = lv;
    *step = (double)pow(2, lv);
    *block = (unsigned long long)pow(2, lv - time_block);
}

double oracle_energy(int n, const double *x, const double *v, const double *mass,
                     double eps2, int nthreads) {
    double *pot = (double *)malloc(sizeof(double) * (n > 0 ? n : 1));
    set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < n; ++i) {
        double w = 0.0;
        for (int j = i + 1; j < n; ++j) {
            double r2 = eps2;
            for (int d = 0; d < 3; ++d) {
                const double dx = x[3 * j + d] - x[3 * i + d];
                r2 += dx * dx;
            }
            w += mass[j] / sqrt(r2);
        }
        pot[i] = -mass[i] * w;
    }
    double e = 0.0;
    for (int i = 0; i < n; ++i) {
        const double v2 = v[3 * i] * v[3 * i] + v[3 * i + 1] * v[3 * i + 1] + v[3 * i + 2] * v[3 * i + 2];
        e += 0.5 * mass[i] * v2 + pot[i];
    }
    free(pot);
    return e;
}

/* Error scale of the regular sums: for each target, sum over the regular j of
 * |m r^-3 dx| and |m r^-3 (dv - 3 (dx.dv) dx / r^2)| (vector norms).  A sum
 * computed with FP32 pair terms carries an absolute error proportional to
 * these, whatever the cancellation between terms; tests use them as the scale
 * for degenerate inputs (tiny N, R_nb = 0). */
void oracle_reg_scale(int n, const double *px, const double *pv, const double *mass,
                      const double *r2nb, double eps2, int nt, const int *targets,
                      double *acc_abs, double *jerk_abs, int nthreads) {
    set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 4)
    for (int k = 0; k < nt; ++k) {
        const int i = targets[k];
        double sa = 0.0, sj = 0.0;
        for (int j = 0; j < n; ++j) {
            if (j == i) continue;
            double x[3], v[3], r2 = 0.0, vx = 0.0;
            for (int d = 0; d < 3; ++d) {
                x[d] = px[3 * j + d] - px[3 * i + d];
                v[d] = pv[3 * j + d] - pv[3 * i + d];
                r2 += x[d] * x[d];
                vx += v[d] * x[d];
            }
            if (r2 < r2nb[i]) continue;
            const double r2s = r2 + eps2;
            const double m_r3 = mass[j] / r2s / sqrt(r2s);
            double a2 = 0.0, j2 = 0.0;
            for (int d = 0; d < 3; ++d) {
                const double a = m_r3 * x[d];
                const double jj = m_r3 * (v[d] - 3 * x[d] * vx / r2s);
                a2 += a * a;
                j2 += jj * jj;
            }
            sa += sqrt(a2);
            sj += sqrt(j2);
        }
        acc_abs[k] = sa;
        jerk_abs[k] = sj;
    }
}

/* CalculateAcceleration23, src_mpi/Particle/Initialize.cpp:102-185: the same
 * expressions in the same order (a21, a21dot, rdf_r2, vdf_r2, rdfdot_r2, then
 * a, b, c, then adot2, adot3 per dimension). */
void oracle_init_derivs23(int n, const double *x, const double *v, const double *mass,
                          const double *r2nb, const double *a0, const double *a1, double eps2,
                          int nt, const int *targets, double *reg2, double *reg3, double *irr2,
                          double *irr3, int nthreads) {
    set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 4)
    for (int k = 0; k < nt; ++k) {
        const int i = targets[k];
        double r2o[3] = {0, 0, 0}, r3o[3] = {0, 0, 0}, i2o[3] = {0, 0, 0}, i3o[3] = {0, 0, 0};
        double a1i[3], a1doti[3];
        for (int d = 0; d < 3; ++d) {
            a1i[d] = a0[3 * i + d];
            a1doti[d] = a1[3 * i + d];
        }
        for (int j = 0; j < n; ++j) {
            if (j == i) continue;
            double xx[3], vv[3], a21[3], a21dot[3];
            double r2u = 0.0, vr = 0.0, v2 = 0.0, rdf_r2 = 0.0, vdf_r2 = 0.0, rdfdot_r2 = 0.0;
            for (int d = 0; d < 3; ++d) {
                xx[d] = x[3 * j + d] - x[3 * i + d];
                vv[d] = v[3 * j + d] - v[3 * i + d];
                r2u += xx[d] * xx[d];
                vr += vv[d] * xx[d];
                v2 += vv[d] * vv[d];
            }
            const double r2 = r2u + eps2;
            const double r3 = r2 * sqrt(r2);
            const double m_r3 = mass[j] / r3;
            for (int d = 0; d < 3; ++d) {
                a21[d] = m_r3 * xx[d];
                a21dot[d] = m_r3 * (vv[d] - 3 * xx[d] * vr / r2);
                rdf_r2 += xx[d] * (a1i[d] - a0[3 * j + d]) / r2;
                vdf_r2 += vv[d] * (a1i[d] - a0[3 * j + d]) / r2;
                rdfdot_r2 += xx[d] * (a1doti[d] - a1[3 * j + d]) / r2;
            }
            const double a = vr / r2;
            const double b = v2 / r2 + rdf_r2 + a * a;
            const double c = 3 * vdf_r2 + rdfdot_r2 + a * (3 * b - 4 * a * a);
            const int reg = !(r2u < r2nb[i]);
            for (int d = 0; d < 3; ++d) {
                const double adot2 = -mass[j] * (a1i[d] - a0[3 * j + d]) / r3 - 6 * a * a21dot[d] - 3 * b * a21[d];
                const double adot3 = -mass[j] * (a1doti[d] - a1[3 * j + d]) / r3 - 9 * a * adot2 -
                                     9 * b * a21dot[d] - 3 * c * a21[d];
                if (reg) {
                    r2o[d] += adot2;
                    r3o[d] += adot3;
                } else {
                    i2o[d] += adot2;
                    i3o[d] += adot3;
                }
            }
        }
        for (int d = 0; d < 3; ++d) {
            reg2[3 * k + d] = r2o[d];
            reg3[3 * k + d] = r3o[d];
            irr2[3 * k + d] = i2o[d];
            irr3[3 * k + d] = i3o[d];
        }
    }
}
