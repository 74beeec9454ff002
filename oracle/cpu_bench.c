/*
 * CPU timing drivers for the reference's own paths of the benchmark
 * configurations, run over a batch of instances with POSIX threads (the
 * library is single-threaded and reentrant on the panel-major path, so
 * instances are distributed over threads, instance i to thread i % nthreads):
 *   cpu_posv_batch     SPD solve chain dpotrf_l + dtrsv_lnn + dtrsv_ltn;
 *   cpu_chain_batch    n = 16 chain dsyrk_ln + ddiare + dpotrf_l + dtrsm_rltn +
 *                      dgemm_nt;
 *   cpu_ric_trf_batch  Riccati factorization, dpotrf_l then per stage
 *                      dtrmm_rlnn + dsyrk_dpotrf_ln
 *                      (examples/example_d_riccati_recursion.c:115-143).
 *
 * TEST / BASELINE INFRASTRUCTURE ONLY: bench.py's CPU-baseline leg and
 * `--impl reference` arm call it with function pointers into either the
 * compiled reference (oracle/_ref/libblasfeo_ref_*.so, symbols blasfeo_*) or
 * the oracle restatement (liboracle.so, symbols oracle_d_*).  Descriptors use
 * the BLASFEO struct layout (include/blasfeo_common.h:67-110).
 */
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

struct dm { double *mem, *pA, *dA; int m, n, pm, cn, use_dA, memsize; };
struct dv { double *mem, *pa; int m, pm, memsize; };
typedef void (*potrf_fn)(int, struct dm *, int, int, struct dm *, int, int);
typedef void (*trsv_fn)(int, struct dm *, int, int, struct dv *, int, struct dv *, int);

struct job {
	int t, nt, num, max_n;
	const int *n;
	struct dm *A;
	struct dv *b, *x;
	potrf_fn potrf;
	trsv_fn lnn, ltn;
};

/* layout of blasfeo_create_dmat (auxiliary/d_aux_lib4.c:1548) */
static void make_mat(int m, struct dm *s, double *mem)
{
	int pm = (m + 3) / 4 * 4;
	s->mem = mem; s->pA = mem; s->dA = mem + (size_t)pm * pm;
	s->m = m; s->n = m; s->pm = pm; s->cn = pm; s->use_dA = 0;
	s->memsize = (int)(((size_t)pm * pm + (m + 15) / 16 * 16) * sizeof(double));
}

static void *worker(void *p)
{
	struct job *j = (struct job *)p;
	int pmax = (j->max_n + 3) / 4 * 4;
	size_t lbytes = ((size_t)pmax * pmax + pmax + 64) * sizeof(double);
	double *lmem = NULL, *ymem = NULL;
	if (posix_memalign((void **)&lmem, 64, lbytes) || posix_memalign((void **)&ymem, 64, (pmax + 8) * sizeof(double)))
		return NULL;
	memset(lmem, 0, lbytes);
	for (int i = j->t; i < j->num; i += j->nt) {
		int n = j->n[i];
		struct dm L;
		struct dv y;
		make_mat(n, &L, lmem);
		y.mem = ymem; y.pa = ymem; y.m = n; y.pm = (n + 3) / 4 * 4; y.memsize = y.pm * 8;
		j->potrf(n, &j->A[i], 0, 0, &L, 0, 0);
		j->lnn(n, &L, 0, 0, &j->b[i], 0, &y, 0);
		j->ltn(n, &L, 0, 0, &y, 0, &j->x[i], 0);
	}
	free(lmem);
	free(ymem);
	return NULL;
}

/* returns wall seconds for solving all `num` systems with `nthreads` threads */
double cpu_posv_batch(int nthreads, int num, int max_n, const int *n, struct dm *A, struct dv *b, struct dv *x,
                      void *potrf, void *lnn, void *ltn)
{
	if (nthreads < 1) nthreads = 1;
	pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * nthreads);
	struct job *jobs = (struct job *)malloc(sizeof(struct job) * nthreads);
	struct timespec t0, t1;
	clock_gettime(CLOCK_MONOTONIC, &t0);
	for (int t = 0; t < nthreads; t++) {
		jobs[t].t = t; jobs[t].nt = nthreads; jobs[t].num = num; jobs[t].max_n = max_n; jobs[t].n = n;
		jobs[t].A = A; jobs[t].b = b; jobs[t].x = x;
		jobs[t].potrf = (potrf_fn)potrf; jobs[t].lnn = (trsv_fn)lnn; jobs[t].ltn = (trsv_fn)ltn;
		pthread_create(&th[t], NULL, worker, &jobs[t]);
	}
	for (int t = 0; t < nthreads; t++) pthread_join(th[t], NULL);
	clock_gettime(CLOCK_MONOTONIC, &t1);
	free(th);
	free(jobs);
	return (double)(t1.tv_sec - t0.tv_sec) + 1e-9 * (double)(t1.tv_nsec - t0.tv_nsec);
}


/* ---- generic thread runner: fn(arg, i, thread scratch) for i = t, t + nt, ... ---- */
typedef void (*inst_fn)(void *arg, int i, double *scratch);
struct rjob { int t, nt, num; inst_fn fn; void *arg; size_t scratch; };

static void *rworker(void *p)
{
	struct rjob *j = (struct rjob *)p;
	double *scr = NULL;
	if (posix_memalign((void **)&scr, 64, j->scratch * sizeof(double) + 64)) return NULL;
	memset(scr, 0, j->scratch * sizeof(double) + 64);
	for (int i = j->t; i < j->num; i += j->nt) j->fn(j->arg, i, scr);
	free(scr);
	return NULL;
}

static double run_threads(int nthreads, int num, inst_fn fn, void *arg, size_t scratch)
{
	if (nthreads < 1) nthreads = 1;
	pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * nthreads);
	struct rjob *jobs = (struct rjob *)malloc(sizeof(struct rjob) * nthreads);
	struct timespec t0, t1;
	clock_gettime(CLOCK_MONOTONIC, &t0);
	for (int t = 0; t < nthreads; t++) {
		jobs[t].t = t; jobs[t].nt = nthreads; jobs[t].num = num; jobs[t].fn = fn; jobs[t].arg = arg;
		jobs[t].scratch = scratch;
		pthread_create(&th[t], NULL, rworker, &jobs[t]);
	}
	for (int t = 0; t < nthreads; t++) pthread_join(th[t], NULL);
	clock_gettime(CLOCK_MONOTONIC, &t1);
	free(th);
	free(jobs);
	return (double)(t1.tv_sec - t0.tv_sec) + 1e-9 * (double)(t1.tv_nsec - t0.tv_nsec);
}

/* an m x n matrix laid out by blasfeo_create_dmat at mem (auxiliary/d_aux_lib4.c:1548) */
static void make_mat_mn(int m, int n, struct dm *s, double *mem)
{
	int pm = (m + 3) / 4 * 4, cn = (n + 3) / 4 * 4, mn = m < n ? m : n;
	s->mem = mem; s->pA = mem; s->dA = mem + (size_t)pm * cn;
	s->m = m; s->n = n; s->pm = pm; s->cn = cn; s->use_dA = 0;
	s->memsize = (int)((((size_t)pm * cn + (mn + 15) / 16 * 16) * sizeof(double) + 63) / 64 * 64);
}

typedef void (*syrk_fn)(int, int, double, struct dm *, int, int, struct dm *, int, int, double, struct dm *, int, int,
                        struct dm *, int, int);
typedef void (*gemm_fn)(int, int, int, double, struct dm *, int, int, struct dm *, int, int, double, struct dm *, int,
                        int, struct dm *, int, int);
typedef void (*diare_fn)(int, double, struct dm *, int, int);
typedef void (*trsm_fn)(int, int, double, struct dm *, int, int, struct dm *, int, int, struct dm *, int, int);
typedef void (*syrk_potrf_fn)(int, int, struct dm *, int, int, struct dm *, int, int, struct dm *, int, int,
                              struct dm *, int, int);

/* ---- n = 16 chain: S = A A^T + shift I, L = chol(S), X = R L^{-T}, D = C - X G^T ---- */
struct chain_arg {
	int k; double shift;
	double *A, *R, *C, *G, *L, *X, *D;
	long long sa, sr, sc, sg, sl, sx, sd;
	syrk_fn syrk; diare_fn diare; potrf_fn potrf; trsm_fn trsm; gemm_fn gemm;
};

static void chain_one(void *p, int i, double *scr)
{
	struct chain_arg *a = (struct chain_arg *)p;
	struct dm A, R, C, G, L, X, D, S;
	make_mat_mn(16, a->k, &A, a->A + a->sa * i);
	make_mat_mn(16, 16, &R, a->R + a->sr * i);
	make_mat_mn(16, 16, &C, a->C + a->sc * i);
	make_mat_mn(16, 16, &G, a->G + a->sg * i);
	make_mat_mn(16, 16, &L, a->L + a->sl * i);
	make_mat_mn(16, 16, &X, a->X + a->sx * i);
	make_mat_mn(16, 16, &D, a->D + a->sd * i);
	make_mat_mn(16, 16, &S, scr);
	a->syrk(16, a->k, 1.0, &A, 0, 0, &A, 0, 0, 0.0, &S, 0, 0, &S, 0, 0);
	a->diare(16, a->shift, &S, 0, 0);
	a->potrf(16, &S, 0, 0, &L, 0, 0);
	a->trsm(16, 16, 1.0, &L, 0, 0, &R, 0, 0, &X, 0, 0);
	a->gemm(16, 16, 16, -1.0, &X, 0, 0, &G, 0, 0, 1.0, &C, 0, 0, &D, 0, 0);
}

/* slabs of `num` instances, instance i of slab P at P + sP*i (elements); returns wall seconds */
double cpu_chain_batch(int nthreads, int num, int k, double shift, double *A, long long sa, double *R, long long sr,
                       double *C, long long sc, double *G, long long sg, double *L, long long sl, double *X,
                       long long sx, double *D, long long sd, void *syrk, void *diare, void *potrf, void *trsm,
                       void *gemm)
{
	struct chain_arg a = {k, shift, A, R, C, G, L, X, D, sa, sr, sc, sg, sl, sx, sd,
	                      (syrk_fn)syrk, (diare_fn)diare, (potrf_fn)potrf, (trsm_fn)trsm, (gemm_fn)gemm};
	return run_threads(nthreads, num, chain_one, &a, 16 * 16 + 16);
}

/* ---- Riccati factorization (LQR backward pass), stage sizes nu + nx <= 16 ----
 * BAbt: batch*N instances 16 x nx (problem b, stage k at b*N + k), RSQ and L:
 * batch*(N+1) instances 16 x 16 (problem b, stage k at b*(N+1) + k). */
struct ric_arg {
	int N, nx, nu;
	double *BA, *RSQ, *L;
	long long sba, srsq, sl;
	potrf_fn potrf; trsm_fn trmm; syrk_potrf_fn syrk_potrf;
};

static void ric_one(void *p, int b, double *scr)
{
	struct ric_arg *a = (struct ric_arg *)p;
	const int N = a->N, nx = a->nx, nu = a->nu, m = nu + nx;
	struct dm Q, LN, W;
	make_mat_mn(16, 16, &Q, a->RSQ + a->srsq * ((long long)b * (N + 1) + N));
	make_mat_mn(16, 16, &LN, a->L + a->sl * ((long long)b * (N + 1) + N));
	make_mat_mn(16, nx, &W, scr);
	a->potrf(nx, &Q, 0, 0, &LN, 0, 0);
	for (int k = N - 1; k >= 0; k--) {
		struct dm BA, R, Lk, Lk1;
		make_mat_mn(16, nx, &BA, a->BA + a->sba * ((long long)b * N + k));
		make_mat_mn(16, 16, &R, a->RSQ + a->srsq * ((long long)b * (N + 1) + k));
		make_mat_mn(16, 16, &Lk, a->L + a->sl * ((long long)b * (N + 1) + k));
		make_mat_mn(16, 16, &Lk1, a->L + a->sl * ((long long)b * (N + 1) + k + 1));
		const int off = (k + 1 == N) ? 0 : nu;
		a->trmm(m, nx, 1.0, &Lk1, off, off, &BA, 0, 0, &W, 0, 0);
		a->syrk_potrf(m, nx, &W, 0, 0, &W, 0, 0, &R, 0, 0, &Lk, 0, 0);
	}
}

double cpu_ric_trf_batch(int nthreads, int batch, int N, int nx, int nu, double *BA, long long sba, double *RSQ,
                         long long srsq, double *L, long long sl, void *potrf, void *trmm, void *syrk_potrf)
{
	struct ric_arg a = {N, nx, nu, BA, RSQ, L, sba, srsq, sl, (potrf_fn)potrf, (trsm_fn)trmm,
	                    (syrk_potrf_fn)syrk_potrf};
	return run_threads(nthreads, batch, ric_one, &a, 16 * ((nx + 3) / 4 * 4) + 16);
}

/* ---- one batched launch of the mixed-op stream: gemm_nt (D = A B^T),
 * potrf_l, getrf_rp, geqrf per instance (descriptor arrays in host memory,
 * instance i of A / B / D at A[i], B[i], D[i]) ---- */
typedef void (*getrf_fn)(int, int, struct dm *, int, int, struct dm *, int, int, int *);
typedef int (*geqrf_ws_fn)(int, int);
typedef void (*geqrf_fn)(int, int, struct dm *, int, int, struct dm *, int, int, void *);
struct ops_arg {
	int op;
	const int *m, *n, *k;
	struct dm *A, *B, *D;
	gemm_fn gemm; potrf_fn potrf; getrf_fn getrf; geqrf_ws_fn geqrf_ws; geqrf_fn geqrf;
};

static void ops_one(void *p, int i, double *scr)
{
	struct ops_arg *a = (struct ops_arg *)p;
	const int m = a->m[i], n = a->n[i];
	switch (a->op) {
	case 0: a->gemm(m, n, a->k[i], 1.0, &a->A[i], 0, 0, &a->B[i], 0, 0, 0.0, &a->D[i], 0, 0, &a->D[i], 0, 0); break;
	case 1: a->potrf(n, &a->A[i], 0, 0, &a->D[i], 0, 0); break;
	case 2: a->getrf(m, n, &a->A[i], 0, 0, &a->D[i], 0, 0, (int *)scr); break;
	default: a->geqrf(m, n, &a->A[i], 0, 0, &a->D[i], 0, 0, scr + 512); break;
	}
}

/* scratch per thread: pivots (512 ints) then the geqrf work buffer */
double cpu_ops_batch(int nthreads, int op, int batch, const int *m, const int *n, const int *k, struct dm *A,
                     struct dm *B, struct dm *D, void *gemm, void *potrf, void *getrf, void *geqrf_ws, void *geqrf,
                     int max_m, int max_n)
{
	struct ops_arg a = {op, m, n, k, A, B, D, (gemm_fn)gemm, (potrf_fn)potrf, (getrf_fn)getrf,
	                    (geqrf_ws_fn)geqrf_ws, (geqrf_fn)geqrf};
	size_t ws = 1024;
	if (op == 3 && geqrf_ws) ws += (size_t)((geqrf_ws_fn)geqrf_ws)(max_m, max_n) / sizeof(double) + 64;
	return run_threads(nthreads, batch, ops_one, &a, ws);
}
