/*
 * CPU oracle for the BLASFEO level-3 / LAPACK hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py load this library, and only as the checker.
 * The product (blasfeo_b200) never links or calls it.
 *
 * It restates, with plain loops, the arithmetic of BLASFEO 0.1.4.2
 * (LA=HIGH_PERFORMANCE, MF=PANELMAJ, panel size 4 for double and single); see
 * oracle_x.h for the per-routine citations.  The restatement is pinned against
 * the compiled reference (oracle/_ref, built by oracle/Makefile) by
 * tests/test_oracle.py, and against the committed golden fixtures generated
 * from that compiled reference (tests/golden/make_golden.py).
 */
#include <math.h>
#include <stddef.h>

struct oracle_dmat { double *mem; double *pA; double *dA; int m, n, pm, cn, use_dA, memsize; };
struct oracle_smat { float *mem; float *pA; float *dA; int m, n, pm, cn, use_dA, memsize; };
struct oracle_dvec { double *mem; double *pa; int m, pm, memsize; };
struct oracle_svec { float *mem; float *pa; int m, pm, memsize; };

#define REAL double
#define OX(name) oracle_d_##name
#define XMAT oracle_dmat
#define XVEC oracle_dvec
#define SQRTX sqrt
#include "oracle_x.h"
#undef REAL
#undef OX
#undef XMAT
#undef XVEC
#undef SQRTX

#define REAL float
#define OX(name) oracle_s_##name
#define XMAT oracle_smat
#define XVEC oracle_svec
#define SQRTX sqrtf
#include "oracle_x.h"
#undef REAL
#undef OX
#undef XMAT
#undef XVEC
#undef SQRTX
