/*
 * TEST INFRASTRUCTURE ONLY: the bandwidth-bound steps of eT's CCSD residual restated in C with
 * OpenMP, for the CPU restatement of eT's algorithm (oracle/et_cpu.py) that the benchmark times
 * as its CPU baseline.  eT runs these steps as OpenMP loops over its arrays; restating them in C
 * keeps the CPU baseline's reorders on all host cores, as eT's are.  Nothing in the product
 * library links or calls this file.
 *
 * Conventions (eT's, 0-based): doubles packed over (ai, bj), ai = a + nv*i, element
 * max(ai,bj)(max(ai,bj)+1)/2 + min(ai,bj) (src/tools/reordering.F90:4174-4198).  Pair indices of
 * the +/- ladder: p(i,j) = i(i+1)/2 + j for i >= j, m(i,j) = i(i-1)/2 + j for i > j.
 */
#include <stdint.h>

static inline int64_t pk(int64_t x, int64_t y) {
    const int64_t M = x > y ? x : y, m = x > y ? y : x;
    return M * (M + 1) / 2 + m;
}

/* squareup_real (reordering.F90:4174): full[r + n c] = packed[pk(r, c)], n = nov */
void et_squareup(const double *packed, double *full, int64_t n) {
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < n; c++) {
        double *col = full + c * n;
        const int64_t cc = c * (c + 1) / 2;
        for (int64_t r = 0; r <= c; r++) col[r] = packed[cc + r];
        for (int64_t r = c + 1; r < n; r++) col[r] = packed[r * (r + 1) / 2 + c];
    }
}

/* packed[pk(M, m)] += alpha * (full[m + n M] + sym * full[M + n m]) * (1/2 if M == m), M >= m:
 * packin after scale_diagonal(1/2) (reordering.F90:4267, omega_ccsd.F90:100-102); sym = 1 also
 * folds in symmetric_sum (reordering.F90:416) */
void et_pack_half(const double *full, double *packed, int64_t n, double alpha, int sym) {
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t M = 0; M < n; M++) {
        double *row = packed + M * (M + 1) / 2;
        const double *colM = full + M * n;
        for (int64_t m = 0; m <= M; m++) {
            double v = colM[m];
            if (sym) v += full[M + n * m];
            if (m == M) v *= 0.5;
            row[m] += alpha * v;
        }
    }
}

/* out (contiguous, dims n[0..3], dim 0 fastest) = alpha * in[i0 s0 + i1 s1 + i2 s2 + i3 s3]
 * + beta * out: eT's sort_* / add_*_to_1234 routines (reordering.F90) */
void et_permute4(const double *in, const int64_t *s, double *out, const int64_t *n, double alpha, double beta) {
    const int64_t n0 = n[0], n1 = n[1], n2 = n[2], n3 = n[3];
#pragma omp parallel for collapse(2) schedule(static)
    for (int64_t i3 = 0; i3 < n3; i3++) {
        for (int64_t i2 = 0; i2 < n2; i2++) {
            const double *src = in + i2 * s[2] + i3 * s[3];
            double *dst = out + n0 * n1 * (i2 + n2 * i3);
            for (int64_t b1 = 0; b1 < n1; b1 += 32)
                for (int64_t b0 = 0; b0 < n0; b0 += 32) {
                    const int64_t e1 = b1 + 32 < n1 ? b1 + 32 : n1, e0 = b0 + 32 < n0 ? b0 + 32 : n0;
                    for (int64_t i1 = b1; i1 < e1; i1++)
                        for (int64_t i0 = b0; i0 < e0; i0++) {
                            const double v = alpha * src[i0 * s[0] + i1 * s[1]];
                            double *o = dst + i0 + n0 * i1;
                            *o = beta != 0.0 ? v + beta * *o : v;
                        }
                }
        }
    }
}

/* construct_plus_minus_2413_from_packed (packed_array_utilities_r.F90:140) with
 * scale_double_packed_blocks(p_factor = q_factor = 1/2) (omega_ccsd.F90:203-210):
 *   tp[p(i,j) + nop p(c,d)] = (1 - d_cd/2)(1 - d_ij/2)(t_cidj + t_cjdi),  i >= j, c >= d
 *   tm[m(i,j) + nom m(c,d)] = t_cidj - t_cjdi,                           i > j,  c > d
 * t_aibj from the packed doubles t2p.  Column-major (nop x nvp) and (nom x nvm). */
void et_t_pm(const double *t2p, int64_t no, int64_t nv, double *tp, double *tm) {
    const int64_t nop = no * (no + 1) / 2, nom = no * (no - 1) / 2;
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t c = 0; c < nv; c++) {
        for (int64_t d = 0; d <= c; d++) {
            const int64_t cdp = c * (c + 1) / 2 + d, cdm = c * (c - 1) / 2 + d;
            for (int64_t i = 0; i < no; i++) {
                for (int64_t j = 0; j <= i; j++) {
                    const double x = t2p[pk(c + nv * i, d + nv * j)], y = t2p[pk(c + nv * j, d + nv * i)];
                    double v = x + y;
                    if (c == d) v *= 0.5;
                    if (i == j) v *= 0.5;
                    tp[i * (i + 1) / 2 + j + nop * cdp] = v;
                    if (c > d && i > j) tm[i * (i - 1) / 2 + j + nom * cdm] = x - y;
                }
            }
        }
    }
}

/* construct_plus_minus_1324_from_full / _from_RFP (packed_array_utilities_r.F90:200, :290) for one
 * (a, b) batch pair: G[((al nv + c) lb + bl) nv + d] = g_acbd for a = a0 + al, b = b0 + bl (the
 * C-order result of L_A L_B^T).  For the npair pairs (pa[k], pb[k]) (a >= b) of the batch:
 *   gp[k + npair p(c,d)] = g_acbd + g_adbc   (c >= d)
 *   gm[k + npair m(c,d)] = g_acbd - g_adbc   (c > d)
 * i.e. row-major (npair x nvp) and (npair x nvm), the transposes of eT's g+_cd,ab and g-_cd,ab. */
void et_g_pm_block(const double *G, int64_t nv, int64_t a0, int64_t b0, int64_t lb, int64_t npair,
                   const int64_t *pa, const int64_t *pb, double *gp, double *gm) {
    const int64_t nvp = nv * (nv + 1) / 2, nvm = nv * (nv - 1) / 2;
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < npair; k++) {
        const int64_t al = pa[k] - a0, bl = pb[k] - b0;
        const double *g = G + (al * nv * lb + bl) * nv;   /* g[c * lb nv + d] = g_acbd */
        const int64_t ldc = lb * nv;
        double *rp = gp + k * nvp, *rm = gm + k * nvm;
        for (int64_t c = 0; c < nv; c++) {
            const double *gc = g + c * ldc;
            for (int64_t d = 0; d <= c; d++) {
                const double x = gc[d], y = g[d * ldc + c];
                rp[c * (c + 1) / 2 + d] = x + y;
                if (c > d) rm[c * (c - 1) / 2 + d] = x - y;
            }
        }
    }
}

/* add_double_packed_plus_minus / add_single_packed_plus_minus (packed_array_utilities_r.F90:335,
 * :402) after scale_double_packed_blocks(q_factor = 1/2): for the pairs (a, b) = (pa[k], pb[k]),
 * with wp[p(i,j) + nop k] and wm[m(i,j) + nom k] (column-major (nop x npair), (nom x npair)),
 *   w+ = wp (1/2 if a == b);   x1 = w+ + w-, x2 = w+ - w- (w- = 0 if i == j or a == b)
 *   om2[pk(a + nv i, b + nv j)] += x1,   om2[pk(a + nv j, b + nv i)] += x2.
 * Every packed element touched by pair k belongs to pair k alone, so pairs run in parallel. */
void et_add_pm(double *om2, const double *wp, const double *wm, int64_t no, int64_t nv, int64_t npair,
               const int64_t *pa, const int64_t *pb) {
    const int64_t nop = no * (no + 1) / 2, nom = no * (no - 1) / 2;
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < npair; k++) {
        const int64_t a = pa[k], b = pb[k];
        const double *cp = wp + nop * k, *cm = wm + nom * k;
        for (int64_t i = 0; i < no; i++) {
            for (int64_t j = 0; j <= i; j++) {
                double w = cp[i * (i + 1) / 2 + j];
                if (a == b) w *= 0.5;
                const double m = (i != j && a != b) ? cm[i * (i - 1) / 2 + j] : 0.0;
                om2[pk(a + nv * i, b + nv * j)] += w + m;
                om2[pk(a + nv * j, b + nv * i)] += w - m;
            }
        }
    }
}
