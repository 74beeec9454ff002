/*
 * CPU timing driver for the SPD solve chain (dpotrf_l + dtrsv_lnn + dtrsv_ltn)
 * of BLASFEO: the reference's own path, run over a batch of systems with
 * POSIX threads (the library is single-threaded and reentrant on the
 * panel-major path, so instances are distributed over threads).
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
