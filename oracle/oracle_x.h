/*
 * Oracle body, instantiated once for double (prefix oracle_d) and once for
 * float (prefix oracle_s) by oracle.c.  TEST INFRASTRUCTURE ONLY: this is the
 * CPU checker that tests/, smoke() and the CPU-baseline leg of bench.py call;
 * the product never links it.
 *
 * Every routine restates the arithmetic of BLASFEO 0.1.4.2 (LA=HIGH_PERFORMANCE,
 * MF=PANELMAJ, ps=4) on host panel-major storage, with plain loops.  Citations
 * are relative to the BLASFEO source tree.
 *
 * Macros expected from the includer:  REAL, OX(name) (name mangling), XMAT (the
 * matrix struct type), XVEC (the vector struct type), SQRTX (sqrt for REAL).
 */

/* element (i,j) of a panel-major matrix, panel size 4:
 * include/blasfeo_common.h:112 (BLASFEO_DMATEL) */
#define EL(sA, i, j) ((sA)->pA[((i) - ((i) & 3)) * (sA)->cn + (j) * 4 + ((i) & 3)])

/* ---- storage: auxiliary/d_aux_lib4.c:1519 (memsize), :1548 (create) ---- */
size_t OX(memsize_mat)(int m, int n)
{
	int pm = (m + 3) / 4 * 4;
	int cn = (n + 3) / 4 * 4;
	int mn = m < n ? m : n;
	int dl = (mn + 15) / 16 * 16;          /* al = ps*PLD = 16 */
	size_t sz = ((size_t)pm * cn + dl) * sizeof(REAL);
	return (sz + 63) / 64 * 64;            /* CACHE_LINE_SIZE rounding */
}

void OX(create_mat)(int m, int n, struct XMAT *sA, void *mem)
{
	int pm = (m + 3) / 4 * 4;
	int cn = (n + 3) / 4 * 4;
	int mn = m < n ? m : n;
	int dl = (mn + 15) / 16 * 16;
	sA->mem = (REAL *)mem;
	sA->pA = (REAL *)mem;
	sA->dA = (REAL *)mem + (size_t)pm * cn;
	sA->m = m;
	sA->n = n;
	sA->pm = pm;
	sA->cn = cn;
	sA->use_dA = 0;
	size_t sz = ((size_t)pm * cn + dl) * sizeof(REAL);
	sA->memsize = (int)((sz + 63) / 64 * 64);
}

/* auxiliary/d_aux_lib4.c:1575,1588 */
size_t OX(memsize_vec)(int m) { return (size_t)((m + 3) / 4 * 4) * sizeof(REAL); }

void OX(create_vec)(int m, struct XVEC *sa, void *mem)
{
	sa->mem = (REAL *)mem;
	sa->pa = (REAL *)mem;
	sa->m = m;
	sa->pm = (m + 3) / 4 * 4;
	sa->memsize = sa->pm * (int)sizeof(REAL);
}

/* auxiliary/d_aux_lib4.c:1607 (pack) and :2238 (unpack): column-major <-> panel-major */
void OX(pack_mat)(int m, int n, const REAL *A, int lda, struct XMAT *sA, int ai, int aj)
{
	if (m <= 0 || n <= 0) return;
	sA->use_dA = 0;
	for (int j = 0; j < n; j++)
		for (int i = 0; i < m; i++)
			EL(sA, ai + i, aj + j) = A[i + (size_t)j * lda];
}

void OX(unpack_mat)(int m, int n, struct XMAT *sA, int ai, int aj, REAL *A, int lda)
{
	for (int j = 0; j < n; j++)
		for (int i = 0; i < m; i++)
			A[i + (size_t)j * lda] = EL(sA, ai + i, aj + j);
}

/* include/blasfeo_d_aux.h blasfeo_dgecp: D = C (sub-blocks) */
void OX(gecp)(int m, int n, struct XMAT *sC, int ci, int cj, struct XMAT *sD, int di, int dj)
{
	sD->use_dA = 0;
	for (int j = 0; j < n; j++)
		for (int i = 0; i < m; i++)
			EL(sD, di + i, dj + j) = EL(sC, ci + i, cj + j);
}

/* include/blasfeo_d_aux.h blasfeo_ddiare: add alpha to the diagonal */
void OX(diare)(int kmax, REAL alpha, struct XMAT *sA, int ai, int aj)
{
	sA->use_dA = 0;
	for (int l = 0; l < kmax; l++)
		EL(sA, ai + l, aj + l) += alpha;
}

/* include/blasfeo_d_aux.h blasfeo_drowsw: swap rows ai and ci over kmax columns */
void OX(rowsw)(int kmax, struct XMAT *sA, int ai, int aj, struct XMAT *sC, int ci, int cj)
{
	sA->use_dA = 0;
	sC->use_dA = 0;
	for (int l = 0; l < kmax; l++) {
		REAL t = EL(sA, ai, aj + l);
		EL(sA, ai, aj + l) = EL(sC, ci, cj + l);
		EL(sC, ci, cj + l) = t;
	}
}

/* D = beta*C + alpha*A*B^T.
 * blasfeo_hp_pm/d_blas3_lib4.c:727 (driver), kernel/generic/kernel_dgemm_4x4_lib4.c:46
 * (4x4 kernel: accumulate sum over k first, then D = alpha*sum + beta*C). */
void OX(gemm_nt)(int m, int n, int k, REAL alpha, struct XMAT *sA, int ai, int aj,
                 struct XMAT *sB, int bi, int bj, REAL beta, struct XMAT *sC, int ci, int cj,
                 struct XMAT *sD, int di, int dj)
{
	if (m <= 0 || n <= 0) return;
	sD->use_dA = 0;
	for (int j = 0; j < n; j++)
		for (int i = 0; i < m; i++) {
			REAL c = 0;
			for (int l = 0; l < k; l++)
				c += EL(sA, ai + i, aj + l) * EL(sB, bi + j, bj + l);
			EL(sD, di + i, dj + j) = alpha * c + beta * EL(sC, ci + i, cj + j);
		}
}

/* Lower triangle of D = beta*C + alpha*A*B^T, m x m, inner size k.
 * blasfeo_hp_pm/d_blas3_lib4.c:5400; blasfeo_ref/x_blas3_ref.c:4130 (REF_SYRK_LN).
 * Elements strictly above the diagonal of D are not written. */
void OX(syrk_ln)(int m, int k, REAL alpha, struct XMAT *sA, int ai, int aj,
                 struct XMAT *sB, int bi, int bj, REAL beta, struct XMAT *sC, int ci, int cj,
                 struct XMAT *sD, int di, int dj)
{
	if (m <= 0) return;
	sD->use_dA = 0;
	for (int j = 0; j < m; j++)
		for (int i = j; i < m; i++) {
			REAL c = 0;
			for (int l = 0; l < k; l++)
				c += EL(sA, ai + i, aj + l) * EL(sB, bi + j, bj + l);
			EL(sD, di + i, dj + j) = alpha * c + beta * EL(sC, ci + i, cj + j);
		}
}

/* D = alpha * B * A^{-T}, A lower triangular non-unit (m x n result, A n x n).
 * The inverse diagonal 1/A_jj is cached in sA->dA (use_dA >= n means valid) and
 * the solve multiplies by it instead of dividing:
 * blasfeo_hp_pm/d_blas3_lib4.c:4123-4193; blasfeo_ref/x_blas3_ref.c:1642-1757;
 * kernel/generic/kernel_dgemm_4x4_lib4.c:5970 (kernel_dtrsm_nt_rl_inv_4x4_lib4). */
void OX(trsm_rltn)(int m, int n, REAL alpha, struct XMAT *sA, int ai, int aj,
                   struct XMAT *sB, int bi, int bj, struct XMAT *sD, int di, int dj)
{
	if (m <= 0 || n <= 0) return;
	sD->use_dA = 0;
	REAL *dA = sA->dA;
	if (ai == 0 && aj == 0) {
		if (sA->use_dA < n) {
			for (int l = 0; l < n; l++) dA[l] = (REAL)1.0 / EL(sA, l, l);
			sA->use_dA = n;
		}
	} else {
		for (int l = 0; l < n; l++) dA[l] = (REAL)1.0 / EL(sA, ai + l, aj + l);
		sA->use_dA = 0;
	}
	for (int j = 0; j < n; j++) {
		REAL inv = dA[j];
		for (int i = 0; i < m; i++) {
			REAL c = alpha * EL(sB, bi + i, bj + j);
			for (int l = 0; l < j; l++)
				c -= EL(sD, di + i, dj + l) * EL(sA, ai + j, aj + l);
			EL(sD, di + i, dj + j) = c * inv;
		}
	}
}

/* Cholesky, lower: D = chol(C) (m x m), left-looking.  Pivot rule from the HP
 * 4x4 kernel (kernel/generic/kernel_dgemm_4x4_lib4.c:5678-5785): if c > 0 then
 * L_jj = sqrt(c), inv = 1/L_jj, else L_jj = 0, inv = 0 (no error).  inv is
 * stored in sD->dA[j]; off-diagonal entries are multiplied by inv.
 * use_dA = m when di == dj == 0 (blasfeo_hp_pm/d_lapack_lib4.c:947-950).
 * Only the lower triangle of D is written. */
void OX(potrf_l)(int m, struct XMAT *sC, int ci, int cj, struct XMAT *sD, int di, int dj)
{
	if (m <= 0) return;
	REAL *dD = sD->dA;
	sD->use_dA = (di == 0 && dj == 0) ? m : 0;
	for (int j = 0; j < m; j++) {
		REAL c = EL(sC, ci + j, cj + j);
		for (int l = 0; l < j; l++)
			c -= EL(sD, di + j, dj + l) * EL(sD, di + j, dj + l);
		REAL d, inv;
		if (c > 0) { d = SQRTX(c); inv = (REAL)1.0 / d; }
		else { d = 0; inv = 0; }
		EL(sD, di + j, dj + j) = d;
		dD[j] = inv;
		for (int i = j + 1; i < m; i++) {
			REAL e = EL(sC, ci + i, cj + j);
			for (int l = 0; l < j; l++)
				e -= EL(sD, di + i, dj + l) * EL(sD, di + j, dj + l);
			EL(sD, di + i, dj + j) = e * inv;
		}
	}
}

/* D = chol(C + A*B^T), lower (m x m, inner size k):
 * blasfeo_hp_pm/d_lapack_lib4.c:1848 (blasfeo_hp_dsyrk_dpotrf_ln),
 * kernel/generic/kernel_dgemm_4x4_lib4.c:5946 (syrk then potrf on the same tile). */
void OX(syrk_potrf_ln)(int m, int k, struct XMAT *sA, int ai, int aj, struct XMAT *sB, int bi, int bj,
                       struct XMAT *sC, int ci, int cj, struct XMAT *sD, int di, int dj)
{
	OX(syrk_ln)(m, k, 1, sA, ai, aj, sB, bi, bj, 1, sC, ci, cj, sD, di, dj);
	OX(potrf_l)(m, sD, di, dj, sD, di, dj);
}

/* LU with row pivoting, P*C = L*U stored in D (unit L below, U on/above).
 * Crout / left-looking column order of blasfeo_ref/x_lapack_ref.c:1156-1530
 * (REF_GETRF_ROWPIVOT) with the pivot rules of the HP kernels
 * (kernel/generic/kernel_dgetrf_pivot_lib4.c:84-165 didamax, :167):
 *   pivot = FIRST row index of the strictly largest |a| in the column;
 *   ipiv[j] = that absolute, 0-based row index; full rows are swapped;
 *   inv = 1/U_jj (0 when U_jj == 0), stored in dA[j]; L entries are a*inv.
 * Columns are processed for j < min(m, n); the remaining columns only get
 * their U part. */
void OX(getrf_rp)(int m, int n, struct XMAT *sC, int ci, int cj, struct XMAT *sD, int di, int dj, int *ipiv)
{
	if (m <= 0 || n <= 0) return;
	REAL *dD = sD->dA;
	sD->use_dA = (di == 0 && dj == 0) ? 1 : 0;
	if (sC != sD || ci != di || cj != dj)
		for (int j = 0; j < n; j++)
			for (int i = 0; i < m; i++)
				EL(sD, di + i, dj + j) = EL(sC, ci + i, cj + j);
	int mn = m < n ? m : n;
	for (int j = 0; j < n; j++) {
		int iu = j < m ? j : m;   /* rows of the U part of this column */
		/* U part: rows 0..iu-1, forward substitution with unit L */
		for (int i = 0; i < iu; i++) {
			REAL u = EL(sD, di + i, dj + j);
			for (int l = 0; l < i; l++)
				u -= EL(sD, di + i, dj + l) * EL(sD, di + l, dj + j);
			EL(sD, di + i, dj + j) = u;
		}
		if (j >= mn) continue;
		/* correct rows j..m-1 and search the pivot */
		REAL amax = -1;
		int ip = j;
		for (int i = j; i < m; i++) {
			REAL a = EL(sD, di + i, dj + j);
			for (int l = 0; l < j; l++)
				a -= EL(sD, di + i, dj + l) * EL(sD, di + l, dj + j);
			EL(sD, di + i, dj + j) = a;
			REAL t = a > 0 ? a : -a;
			if (t > amax) { amax = t; ip = i; }
		}
		ipiv[j] = ip;
		if (ip != j)
			for (int l = 0; l < n; l++) {
				REAL t = EL(sD, di + j, dj + l);
				EL(sD, di + j, dj + l) = EL(sD, di + ip, dj + l);
				EL(sD, di + ip, dj + l) = t;
			}
		REAL p = EL(sD, di + j, dj + j);
		REAL inv = p != 0 ? (REAL)1.0 / p : (REAL)0;
		dD[j] = inv;
		for (int i = j + 1; i < m; i++)
			EL(sD, di + i, dj + j) *= inv;
	}
}

/* Lower trapezoid (m x n, element (i,j) for j <= i < m, j < n) of
 * D = beta*C + alpha*A*B^T, inner size k.
 * blasfeo_hp_pm/d_blas3_lib4.c:6459 (blasfeo_hp_dsyrk_ln_mn);
 * blasfeo_ref/x_blas3_ref.c:4229 (REF_SYRK_LN_MN).  use_dA of D invalidated. */
void OX(syrk_ln_mn)(int m, int n, int k, REAL alpha, struct XMAT *sA, int ai, int aj,
                    struct XMAT *sB, int bi, int bj, REAL beta, struct XMAT *sC, int ci, int cj,
                    struct XMAT *sD, int di, int dj)
{
	if (m <= 0 || n <= 0) return;
	sD->use_dA = 0;
	for (int j = 0; j < n; j++)
		for (int i = j; i < m; i++) {
			REAL c = 0;
			for (int l = 0; l < k; l++)
				c += EL(sA, ai + i, aj + l) * EL(sB, bi + j, bj + l);
			EL(sD, di + i, dj + j) = alpha * c + beta * EL(sC, ci + i, cj + j);
		}
}

/* D = alpha * B * A^{-T}, A lower triangular with unit diagonal (the diagonal
 * is not read), m x n result, A n x n.
 * blasfeo_hp_pm/d_blas3_lib4.c:4359 (blasfeo_hp_dtrsm_rltu);
 * blasfeo_ref/x_blas3_ref.c:1760 (REF_TRSM_RLTU).  use_dA of D invalidated. */
void OX(trsm_rltu)(int m, int n, REAL alpha, struct XMAT *sA, int ai, int aj,
                   struct XMAT *sB, int bi, int bj, struct XMAT *sD, int di, int dj)
{
	if (m <= 0 || n <= 0) return;
	sD->use_dA = 0;
	for (int j = 0; j < n; j++)
		for (int i = 0; i < m; i++) {
			REAL c = alpha * EL(sB, bi + i, bj + j);
			for (int l = 0; l < j; l++)
				c -= EL(sD, di + i, dj + l) * EL(sA, ai + j, aj + l);
			EL(sD, di + i, dj + j) = c;
		}
}

/* Cholesky of the m x n lower trapezoid (n clamped to m): the n x n factor of
 * the leading block and rows n..m-1 of the first n columns solved against it
 * (L_ij = (C_ij - sum_l L_il L_jl) / L_jj).  Pivot rule and inverse diagonal as
 * potrf_l; use_dA = 1 when di == dj == 0, else 0, as the reference sets it.
 * blasfeo_hp_pm/d_lapack_lib4.c:1155-1187 (blasfeo_hp_dpotrf_l_mn);
 * blasfeo_ref/x_lapack_ref.c:185 (REF_POTRF_L_MN). */
void OX(potrf_l_mn)(int m, int n, struct XMAT *sC, int ci, int cj, struct XMAT *sD, int di, int dj)
{
	if (m <= 0 || n <= 0) return;
	if (n > m) n = m;
	REAL *dD = sD->dA;
	sD->use_dA = (di == 0 && dj == 0) ? 1 : 0;
	for (int j = 0; j < n; j++) {
		REAL c = EL(sC, ci + j, cj + j);
		for (int l = 0; l < j; l++)
			c -= EL(sD, di + j, dj + l) * EL(sD, di + j, dj + l);
		REAL d, inv;
		if (c > 0) { d = SQRTX(c); inv = (REAL)1.0 / d; }
		else { d = 0; inv = 0; }
		EL(sD, di + j, dj + j) = d;
		dD[j] = inv;
		for (int i = j + 1; i < m; i++) {
			REAL e = EL(sC, ci + i, cj + j);
			for (int l = 0; l < j; l++)
				e -= EL(sD, di + i, dj + l) * EL(sD, di + j, dj + l);
			EL(sD, di + i, dj + j) = e * inv;
		}
	}
}

/* LU without pivoting, C = L*U stored in D (unit L below, U on/above the
 * diagonal); inv = 1/U_jj (no zero test: a zero pivot divides by zero, as
 * REF_GETRF_NOPIVOT does) in dA[j], L entries a*inv; use_dA = 1 when
 * di == dj == 0.  Crout column order as getrf_rp without the pivot search.
 * blasfeo_hp_pm/d_lapack_lib4.c:2078 (blasfeo_hp_dgetrf_np);
 * blasfeo_ref/x_lapack_ref.c (REF_GETRF_NOPIVOT). */
void OX(getrf_np)(int m, int n, struct XMAT *sC, int ci, int cj, struct XMAT *sD, int di, int dj)
{
	if (m <= 0 || n <= 0) return;
	REAL *dD = sD->dA;
	sD->use_dA = (di == 0 && dj == 0) ? 1 : 0;
	if (sC != sD || ci != di || cj != dj)
		for (int j = 0; j < n; j++)
			for (int i = 0; i < m; i++)
				EL(sD, di + i, dj + j) = EL(sC, ci + i, cj + j);
	int mn = m < n ? m : n;
	for (int j = 0; j < n; j++) {
		int iu = j < m ? j : m;
		for (int i = 0; i < iu; i++) {
			REAL u = EL(sD, di + i, dj + j);
			for (int l = 0; l < i; l++)
				u -= EL(sD, di + i, dj + l) * EL(sD, di + l, dj + j);
			EL(sD, di + i, dj + j) = u;
		}
		if (j >= mn) continue;
		for (int i = j; i < m; i++) {
			REAL a = EL(sD, di + i, dj + j);
			for (int l = 0; l < j; l++)
				a -= EL(sD, di + i, dj + l) * EL(sD, di + l, dj + j);
			EL(sD, di + i, dj + j) = a;
		}
		REAL inv = (REAL)1.0 / EL(sD, di + j, dj + j);
		dD[j] = inv;
		for (int i = j + 1; i < m; i++)
			EL(sD, di + i, dj + j) *= inv;
	}
}

/* Workspace bytes of the HP geqrf: blasfeo_hp_pm/d_lapack_lib4.c:3433-3440.  The
 * oracle itself needs none. */
int OX(geqrf_worksize)(int m, int n)
{
	int cm = (m + 3) / 4 * 4;
	int cn = (n + 3) / 4 * 4;
	return 4 * (cm + cn) * (int)sizeof(REAL);
}

/* Householder QR, D = QR of C: R on and above the diagonal, the essential part
 * of each reflector below it (implicit unit head), tau[j] in sD->dA[di+j].
 * Reflector convention of LAPACK dlarfg as restated by
 * blasfeo_ref/x_lapack_ref.c:1551-1620 and kernel/generic/kernel_dgeqrf_4_lib4.c:80-96:
 *   s = sum_{i>j} x_i^2;  s == 0 -> tau = 0, column untouched;
 *   else beta = -sign(alpha) * sqrt(alpha^2 + s) (alpha > 0 -> negative),
 *        tau = (beta - alpha)/beta, v_i = x_i * (1/(alpha - beta)), R_jj = beta.
 * Each reflector is applied at once to the trailing columns:
 *   w = C_j + sum_{i>j} v_i C_ij, C -= tau * v * w. */
void OX(geqrf)(int m, int n, struct XMAT *sC, int ci, int cj, struct XMAT *sD, int di, int dj, void *work)
{
	(void)work;
	if (m <= 0 || n <= 0) return;
	sD->use_dA = 0;
	REAL *tau = sD->dA + di;
	if (sC != sD || ci != di || cj != dj)
		for (int j = 0; j < n; j++)
			for (int i = 0; i < m; i++)
				EL(sD, di + i, dj + j) = EL(sC, ci + i, cj + j);
	int kmax = m < n ? m : n;
	for (int j = 0; j < kmax; j++) {
		REAL s = 0;
		for (int i = j + 1; i < m; i++) {
			REAL x = EL(sD, di + i, dj + j);
			s += x * x;
		}
		if (s == 0) {
			tau[j] = 0;
		} else {
			REAL alpha = EL(sD, di + j, dj + j);
			REAL beta = SQRTX(s + alpha * alpha);
			if (alpha > 0) beta = -beta;
			tau[j] = (beta - alpha) / beta;
			REAL sc = (REAL)1.0 / (alpha - beta);
			EL(sD, di + j, dj + j) = beta;
			for (int i = j + 1; i < m; i++) EL(sD, di + i, dj + j) *= sc;
		}
		REAL t = tau[j];
		for (int c = j + 1; c < n; c++) {
			REAL w = EL(sD, di + j, dj + c);
			for (int i = j + 1; i < m; i++)
				w += EL(sD, di + i, dj + j) * EL(sD, di + i, dj + c);
			w = -t * w;
			EL(sD, di + j, dj + c) += w;
			for (int i = j + 1; i < m; i++)
				EL(sD, di + i, dj + c) += w * EL(sD, di + i, dj + j);
		}
	}
}

/* D = alpha * B * A, A lower triangular non-unit (right, lower, no-trans):
 * blasfeo_hp_pm/d_blas3_lib4.c:4893 (blasfeo_hp_dtrmm_rlnn), used by the Riccati
 * recursion of examples/example_d_riccati_recursion.c:125. */
void OX(trmm_rlnn)(int m, int n, REAL alpha, struct XMAT *sA, int ai, int aj,
                   struct XMAT *sB, int bi, int bj, struct XMAT *sD, int di, int dj)
{
	if (m <= 0 || n <= 0) return;
	sD->use_dA = 0;
	for (int j = 0; j < n; j++)
		for (int i = 0; i < m; i++) {
			REAL c = 0;
			for (int l = j; l < n; l++)
				c += EL(sB, bi + i, bj + l) * EL(sA, ai + l, aj + j);
			EL(sD, di + i, dj + j) = alpha * c;
		}
}

/* z = A^{-1} x, A lower non-unit (blasfeo_dtrsv_lnn), and z = A^{-T} x
 * (blasfeo_dtrsv_ltn): include/blasfeo_d_blasfeo_api.h; the HP versions use
 * the cached inverse diagonal when valid (blasfeo_hp_pm/d_blas2_lib4.c). */
void OX(trsv_lnn)(int m, struct XMAT *sA, int ai, int aj, struct XVEC *sx, int xi, struct XVEC *sz, int zi)
{
	REAL *x = sx->pa + xi, *z = sz->pa + zi;
	for (int i = 0; i < m; i++) {
		REAL c = x[i];
		for (int l = 0; l < i; l++) c -= EL(sA, ai + i, aj + l) * z[l];
		z[i] = c * ((REAL)1.0 / EL(sA, ai + i, aj + i));
	}
}

void OX(trsv_ltn)(int m, struct XMAT *sA, int ai, int aj, struct XVEC *sx, int xi, struct XVEC *sz, int zi)
{
	REAL *x = sx->pa + xi, *z = sz->pa + zi;
	for (int i = m - 1; i >= 0; i--) {
		REAL c = x[i];
		for (int l = i + 1; l < m; l++) c -= EL(sA, ai + l, aj + i) * z[l];
		z[i] = c * ((REAL)1.0 / EL(sA, ai + i, aj + i));
	}
}

/* z = beta*y + alpha*A*x (blasfeo_dgemv_n). */
void OX(gemv_n)(int m, int n, REAL alpha, struct XMAT *sA, int ai, int aj, struct XVEC *sx, int xi,
                REAL beta, struct XVEC *sy, int yi, struct XVEC *sz, int zi)
{
	for (int i = 0; i < m; i++) {
		REAL c = 0;
		for (int l = 0; l < n; l++) c += EL(sA, ai + i, aj + l) * sx->pa[xi + l];
		sz->pa[zi + i] = alpha * c + beta * sy->pa[yi + i];
	}
}

/* z = beta*y + alpha*A^T*x, A m x n (blasfeo_dgemv_t,
 * blasfeo_hp_pm/d_blas2_lib4.c:113): z_j = beta*y_j + alpha*sum_i A_ij x_i. */
void OX(gemv_t)(int m, int n, REAL alpha, struct XMAT *sA, int ai, int aj, struct XVEC *sx, int xi,
                REAL beta, struct XVEC *sy, int yi, struct XVEC *sz, int zi)
{
	REAL t[512];
	for (int j = 0; j < n; j++) {
		REAL c = 0;
		for (int i = 0; i < m; i++) c += EL(sA, ai + i, aj + j) * sx->pa[xi + i];
		t[j] = alpha * c + beta * sy->pa[yi + j];
	}
	for (int j = 0; j < n; j++) sz->pa[zi + j] = t[j];
}

/* z = A*x and z = A^T*x, A m x m lower non-unit (blasfeo_dtrmv_lnn,
 * blasfeo_dtrmv_ltn; blasfeo_hp_pm/d_blas2_lib4.c:772, :1014); z may alias x. */
void OX(trmv_lnn)(int m, struct XMAT *sA, int ai, int aj, struct XVEC *sx, int xi, struct XVEC *sz, int zi)
{
	REAL t[512];
	for (int i = 0; i < m; i++) {
		REAL c = 0;
		for (int j = 0; j <= i; j++) c += EL(sA, ai + i, aj + j) * sx->pa[xi + j];
		t[i] = c;
	}
	for (int i = 0; i < m; i++) sz->pa[zi + i] = t[i];
}

void OX(trmv_ltn)(int m, struct XMAT *sA, int ai, int aj, struct XVEC *sx, int xi, struct XVEC *sz, int zi)
{
	REAL t[512];
	for (int j = 0; j < m; j++) {
		REAL c = 0;
		for (int i = j; i < m; i++) c += EL(sA, ai + i, aj + j) * sx->pa[xi + i];
		t[j] = c;
	}
	for (int j = 0; j < m; j++) sz->pa[zi + j] = t[j];
}

/* A m x n lower trapezoid (blasfeo_dtrsv_lnn_mn, blasfeo_hp_pm/d_blas2_lib4.c:1275):
 * z[0:n] = A[0:n,0:n]^{-1} x[0:n] (multiplying by the reciprocal pivots),
 * z[n:m] = x[n:m] - A[n:m,0:n] z[0:n]; z may alias x. */
void OX(trsv_lnn_mn)(int m, int n, struct XMAT *sA, int ai, int aj, struct XVEC *sx, int xi, struct XVEC *sz, int zi)
{
	REAL *x = sx->pa + xi, *z = sz->pa + zi;
	if (m < n) m = n;
	for (int i = 0; i < m; i++) {
		REAL c = x[i];
		const int lim = i < n ? i : n;
		for (int l = 0; l < lim; l++) c -= EL(sA, ai + i, aj + l) * z[l];
		z[i] = i < n ? c * ((REAL)1.0 / EL(sA, ai + i, aj + i)) : c;
	}
}

/* A m x n lower trapezoid, transposed (blasfeo_dtrsv_ltn_mn, :1478):
 * z[n:m] = x[n:m]; for i = n-1 .. 0: z[i] = (x[i] - sum_{l>i} A_li z_l) / A_ii. */
void OX(trsv_ltn_mn)(int m, int n, struct XMAT *sA, int ai, int aj, struct XVEC *sx, int xi, struct XVEC *sz, int zi)
{
	REAL *x = sx->pa + xi, *z = sz->pa + zi;
	if (n > m) n = m;
	for (int i = n; i < m; i++) z[i] = x[i];
	for (int i = n - 1; i >= 0; i--) {
		REAL c = x[i];
		for (int l = i + 1; l < m; l++) c -= EL(sA, ai + l, aj + i) * z[l];
		z[i] = c * ((REAL)1.0 / EL(sA, ai + i, aj + i));
	}
}

#undef EL
