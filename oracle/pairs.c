/*
 * C restatement (POSIX threads) of the reference's on-the-fly matrix-vector product
 * (test infrastructure: the timed CPU baseline; never part of the product).
 *
 * Follows src/matrix/matrix_module.f90:
 *   product_q_block_x  (:727-825)  s_q  = T_qq x_q           (Gaussian kernel)
 *   product_mu_block_x (:834-1001) s_q += T_qmu x_mu, s_mu = T_muq x_q + T_mumu x_mu
 *   update_y_q         (:1011-1098) y_q = sum_j c_ij (s_j - s_i), c_ij = K_ij or
 *                                  1/2 (K_ij + (w_j/w_i) K_ji) (heterogeneous)
 *   update_y_mu        (:1107-1125) y_mu = s_mu
 * and new_gmres_diagonal_shift (src/wfq/wfq_module.f90:398-424,
 * src/wfq/wfqfmu_module.f90:698-746): y += D(w) x.
 * As the reference does, each unordered pair i > j is visited once per kernel,
 * threads accumulate into private full-length arrays that are summed at the
 * end, and K is evaluated from the Fermi function for every pair.  The
 * reference uses OpenMP; this image's gcc has no OpenMP runtime, so the same
 * work split (rows dealt cyclically to threads, private accumulators merged
 * at the end) is written with POSIX threads.
 *
 * Build: make -C oracle   (writes oracle/_ref/libplxref.so)
 */
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>
#include <unistd.h>

typedef double complex zc;

#define PLX_PI 3.14159265358979323846

int plxref_max_threads(void);

typedef struct {
    int n_atoms, n_types, fmu, hetero;
    const double *coord;     /* 3 x N bohr */
    const int *type;         /* N */
    const double *rq, *rmu, *eta, *aij;      /* per type */
    const double *fd, *fs, *r0;              /* n_types x n_types, (a,b) at a + nt*b */
    const double *dq;        /* per type: diagonal of the charge rows, complex (re, im) */
    const double *dmu;       /* per atom: diagonal of the dipole rows, complex (re, im) */
    const double *wt;        /* per type: Drude weight w_t, complex (re, im) */
} plxref_sys;

static double fdamp(double r, double R) {
    return erf(r / R) - ((2.0 * r) / (sqrt(PLX_PI) * R)) * exp(-(r * r) / (R * R));
}

static double conductance(const plxref_sys *s, int i, int j, double r) {
    int ti = s->type[i], tj = s->type[j], nt = s->n_types;
    double d = s->fd[ti + nt * tj], sij = s->fs[ti + nt * tj], r0 = s->r0[ti + nt * tj];
    double f = 1.0 / (1.0 + exp(-d * ((r / (sij * r0)) - 1.0)));
    return (1.0 - f) * s->aij[ti] / r;
}

typedef struct {
    const plxref_sys *s;
    const zc *x;
    const zc *S;
    zc *acc;
    int tid, nthr, pass;
} work_t;

static void *pair_worker(void *arg) {
    work_t *w = (work_t *)arg;
    const plxref_sys *s = w->s;
    const int N = s->n_atoms;
    const double *c = s->coord;
    const zc *x = w->x;
    zc *tmp = w->acc;
    for (int i = w->tid; i < N; i += w->nthr) {
        int ti = s->type[i];
        if (w->pass == 0) tmp[i] += s->eta[ti] * x[i];
        for (int j = 0; j < i; ++j) {
            int tj = s->type[j];
            double dx = c[3 * i] - c[3 * j], dy = c[3 * i + 1] - c[3 * j + 1], dz = c[3 * i + 2] - c[3 * j + 2];
            double r = sqrt(dx * dx + dy * dy + dz * dz);
            if (w->pass == 1) {
                const zc *S = w->S;
                double kij = conductance(s, i, j, r);
                if (!s->hetero) {
                    tmp[i] += kij * (S[j] - S[i]);
                    tmp[j] += kij * (S[i] - S[j]);
                } else {
                    double kji = conductance(s, j, i, r);
                    zc wi = s->wt[2 * ti] + I * s->wt[2 * ti + 1], wj = s->wt[2 * tj] + I * s->wt[2 * tj + 1];
                    tmp[i] += 0.5 * (kij + (wj / wi) * kji) * (S[j] - S[i]);
                    tmp[j] += 0.5 * (kji + (wi / wj) * kij) * (S[i] - S[j]);
                }
                continue;
            }
            double qq = erf(r / sqrt(s->rq[ti] * s->rq[ti] + s->rq[tj] * s->rq[tj])) / r;
            tmp[i] += qq * x[j];
            tmp[j] += qq * x[i];
            if (!s->fmu) continue;
            double r3 = r * r * r, r2 = r * r, r5 = r3 * r2;
            const zc *mi = x + N + 3 * i, *mj = x + N + 3 * j;
            zc *ti_mu = tmp + N + 3 * i, *tj_mu = tmp + N + 3 * j;
            double f1 = fdamp(r, sqrt(s->rq[ti] * s->rq[ti] + s->rmu[tj] * s->rmu[tj])) / r3;
            tmp[i] += f1 * (dx * mj[0] + dy * mj[1] + dz * mj[2]);
            tj_mu[0] += f1 * dx * x[i];
            tj_mu[1] += f1 * dy * x[i];
            tj_mu[2] += f1 * dz * x[i];
            double f2 = fdamp(r, sqrt(s->rq[tj] * s->rq[tj] + s->rmu[ti] * s->rmu[ti])) / r3;
            tmp[j] -= f2 * (dx * mi[0] + dy * mi[1] + dz * mi[2]);
            ti_mu[0] -= f2 * dx * x[j];
            ti_mu[1] -= f2 * dy * x[j];
            ti_mu[2] -= f2 * dz * x[j];
            double R = sqrt(s->rmu[ti] * s->rmu[ti] + s->rmu[tj] * s->rmu[tj]);
            double e = exp(-(r * r) / (R * R));
            double fD1 = erf(r / R) - ((2.0 * r) / (sqrt(PLX_PI) * R)) * e;
            double fD2 = (4.0 / (sqrt(PLX_PI) * R * R * R)) * e;
            double d[3] = {dx, dy, dz};
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) {
                    double T = ((-3.0 * d[a] * d[b]) / r5 + (a == b ? 1.0 / r3 : 0.0)) * fD1 + fD2 * d[a] * d[b] / r2;
                    ti_mu[a] += T * mj[b];
                    tj_mu[a] += T * mi[b];
                }
        }
    }
    return NULL;
}

static int run_pass(const plxref_sys *s, const zc *x, const zc *S, zc *out, int len, int pass, int nthr) {
    pthread_t th[256];
    work_t w[256];
    if (nthr < 1) nthr = 1;
    if (nthr > 256) nthr = 256;
    zc *bufs = calloc((size_t)len * nthr, sizeof(zc));
    if (!bufs) return 1;
    for (int t = 0; t < nthr; ++t) {
        w[t] = (work_t){s, x, S, bufs + (size_t)len * t, t, nthr, pass};
        pthread_create(&th[t], NULL, pair_worker, &w[t]);
    }
    for (int t = 0; t < nthr; ++t) pthread_join(th[t], NULL);
    for (int t = 0; t < nthr; ++t)
        for (int k = 0; k < len; ++k) out[k] += bufs[(size_t)len * t + k];
    free(bufs);
    return 0;
}

/* y = A(w) x for one column; x, y complex n_var. */
int plxref_matvec(const plxref_sys *s, const double *xin, double *yout, int n_threads) {
    const int N = s->n_atoms, nv = s->fmu ? 4 * N : N;
    const zc *x = (const zc *)xin;
    zc *y = (zc *)yout;
    zc *S = calloc((size_t)nv, sizeof(zc));
    if (!S) return 1;
    if (n_threads <= 0) n_threads = plxref_max_threads();
    if (run_pass(s, x, NULL, S, nv, 0, n_threads)) return 1;
    memset(y, 0, sizeof(zc) * (size_t)nv);
    if (run_pass(s, x, S, y, N, 1, n_threads)) return 1;
    for (int i = 0; i < N; ++i) {
        int ti = s->type[i];
        y[i] += (s->dq[2 * ti] + I * s->dq[2 * ti + 1]) * x[i];
    }
    if (s->fmu)
        for (int k = N; k < nv; ++k) {
            int i = (k - N) / 3;
            y[k] = S[k] + (s->dmu[2 * i] + I * s->dmu[2 * i + 1]) * x[k];
        }
    free(S);
    return 0;
}

int plxref_max_threads(void) {
    long n = sysconf(_SC_NPROCESSORS_ONLN);
    return n > 0 ? (int)n : 1;
}
