/*
 * Gaussian integrals over primitive Cartesian shells (McMurchie-Davidson).
 *
 * TEST INFRASTRUCTURE ONLY: the molecular front end of the oracle.  eT obtains
 * its AO integrals from Libint 2.7 (src/libint/eri.cpp, oei.cpp), which is not
 * available here; this file restates the textbook McMurchie-Davidson scheme
 * (Hermite expansion coefficients E^{ij}_t, Hermite Coulomb integrals R^n_{tuv}
 * and the Boys function) so that the committed eT test systems can be rebuilt
 * from the cc-pVDZ basis and the CPU oracle pinned against eT's energies.
 *
 * Primitives are unnormalised x^l y^m z^n exp(-a r^2); the caller applies
 * contraction coefficients, normalisation and the Cartesian->spherical map.
 * Shell component order: for total L, (lx, ly, lz) with lx descending, then
 * ly descending (xx, xy, xz, yy, yz, zz for L = 2).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define MAXL 2
#define MAXN (4 * MAXL + 1)

static void boys(int nmax, double T, double *F) {
    if (T < 1e-14) {
        for (int n = 0; n <= nmax; n++) F[n] = 1.0 / (2 * n + 1) - T / (2 * n + 3);
        return;
    }
    if (T < 40.0) {
        /* series for F_nmax, then downward recursion */
        double term = 1.0 / (2 * nmax + 1), sum = term;
        for (int k = 1; k < 400; k++) {
            term *= 2.0 * T / (2 * nmax + 2 * k + 1);
            sum += term;
            if (term < 1e-17 * sum) break;
        }
        double e = exp(-T);
        F[nmax] = e * sum;
        for (int n = nmax; n > 0; n--) F[n - 1] = (2.0 * T * F[n] + e) / (2 * n - 1);
    } else {
        double e = exp(-T);
        F[0] = 0.5 * sqrt(M_PI / T) * erf(sqrt(T));
        for (int n = 0; n < nmax; n++) F[n + 1] = ((2 * n + 1) * F[n] - e) / (2.0 * T);
    }
}

/* E[i][j][t], i <= la, j <= lb + 2 (kinetic needs j+2), t <= i + j */
#define EJ (MAXL + 3)
#define ET (2 * MAXL + 3)
static void hermite_E(int la, int lb, double a, double b, double Ax, double Bx,
                      double E[MAXL + 1][EJ][ET]) {
    double p = a + b, mu = a * b / p, X = Ax - Bx;
    double XPA = -b / p * X, XPB = a / p * X;
    memset(E, 0, sizeof(double) * (MAXL + 1) * EJ * ET);
    E[0][0][0] = exp(-mu * X * X);
    for (int i = 0; i <= la; i++) {
        for (int j = 0; j <= lb; j++) {
            if (i == 0 && j == 0) continue;
            for (int t = 0; t <= i + j; t++) {
                double v = 0.0;
                if (i > 0) {
                    if (t > 0) v += E[i - 1][j][t - 1] / (2 * p);
                    if (t <= i - 1 + j) v += XPA * E[i - 1][j][t];
                    if (t + 1 <= i - 1 + j) v += (t + 1) * E[i - 1][j][t + 1];
                } else {
                    if (t > 0) v += E[i][j - 1][t - 1] / (2 * p);
                    if (t <= i + j - 1) v += XPB * E[i][j - 1][t];
                    if (t + 1 <= i + j - 1) v += (t + 1) * E[i][j - 1][t + 1];
                }
                E[i][j][t] = v;
            }
        }
    }
}

/* R[t][u][v] = R^0_{tuv}(p, PC) for t+u+v <= L */
static void hermite_R(int L, double p, double X, double Y, double Z, double *Rout) {
    static double R[MAXN + 1][MAXN + 1][MAXN + 1][MAXN + 1];
    double F[MAXN + 2];
    double T = p * (X * X + Y * Y + Z * Z);
    boys(L, T, F);
    double f = 1.0;
    for (int n = 0; n <= L; n++) {
        R[n][0][0][0] = f * F[n];
        f *= -2.0 * p;
    }
    for (int n = L - 1; n >= 0; n--) {
        int m = L - n;
        for (int t = 0; t <= m; t++)
            for (int u = 0; u <= m - t; u++)
                for (int v = 0; v <= m - t - u; v++) {
                    if (t + u + v == 0) continue;
                    double val;
                    if (t > 0) {
                        val = X * R[n + 1][t - 1][u][v];
                        if (t > 1) val += (t - 1) * R[n + 1][t - 2][u][v];
                    } else if (u > 0) {
                        val = Y * R[n + 1][t][u - 1][v];
                        if (u > 1) val += (u - 1) * R[n + 1][t][u - 2][v];
                    } else {
                        val = Z * R[n + 1][t][u][v - 1];
                        if (v > 1) val += (v - 1) * R[n + 1][t][u][v - 2];
                    }
                    R[n][t][u][v] = val;
                }
    }
    for (int t = 0; t <= L; t++)
        for (int u = 0; u <= L; u++)
            for (int v = 0; v <= L; v++)
                Rout[(t * (MAXN + 1) + u) * (MAXN + 1) + v] = (t + u + v <= L) ? R[0][t][u][v] : 0.0;
}

static int ncart(int l) { return (l + 1) * (l + 2) / 2; }

static void cart_components(int l, int comp[][3]) {
    int k = 0;
    for (int lx = l; lx >= 0; lx--)
        for (int ly = l - lx; ly >= 0; ly--) {
            comp[k][0] = lx;
            comp[k][1] = ly;
            comp[k][2] = l - lx - ly;
            k++;
        }
}

/* offsets of each primitive shell in the Cartesian primitive basis */
static int *shell_offsets(int nsh, const int *l, int *ntot) {
    int *off = (int *)malloc(sizeof(int) * (nsh + 1));
    off[0] = 0;
    for (int s = 0; s < nsh; s++) off[s + 1] = off[s] + ncart(l[s]);
    *ntot = off[nsh];
    return off;
}

/* one-electron integrals: S, T, V (nuclear attraction over ncent charges) */
void one_electron(int nsh, const int *l, const double *alpha, const double *ctr,
                  int ncent, const double *charges, const double *cpos,
                  double *S, double *Tk, double *V) {
    int n;
    int *off = shell_offsets(nsh, l, &n);
    double Rbuf[(MAXN + 1) * (MAXN + 1) * (MAXN + 1)];
    for (int sa = 0; sa < nsh; sa++)
        for (int sb = 0; sb < nsh; sb++) {
            int la = l[sa], lb = l[sb];
            double a = alpha[sa], b = alpha[sb], p = a + b;
            const double *A = ctr + 3 * sa, *B = ctr + 3 * sb;
            double E[3][MAXL + 1][EJ][ET];
            for (int d = 0; d < 3; d++) hermite_E(la, lb + 2, a, b, A[d], B[d], E[d]);
            int ca[6][3], cb[6][3];
            cart_components(la, ca);
            cart_components(lb, cb);
            double P[3];
            for (int d = 0; d < 3; d++) P[d] = (a * A[d] + b * B[d]) / p;
            double sq = sqrt(M_PI / p);
            for (int ia = 0; ia < ncart(la); ia++)
                for (int ib = 0; ib < ncart(lb); ib++) {
                    double s1[3], t1[3];
                    for (int d = 0; d < 3; d++) {
                        int i = ca[ia][d], j = cb[ib][d];
                        double sij = E[d][i][j][0] * sq;
                        double sij2 = E[d][i][j + 2][0] * sq;
                        double sijm = (j >= 2) ? E[d][i][j - 2][0] * sq : 0.0;
                        s1[d] = sij;
                        t1[d] = -2.0 * b * b * sij2 + b * (2 * j + 1) * sij - 0.5 * j * (j - 1) * sijm;
                    }
                    int row = off[sa] + ia, col = off[sb] + ib;
                    S[row * n + col] = s1[0] * s1[1] * s1[2];
                    Tk[row * n + col] = t1[0] * s1[1] * s1[2] + s1[0] * t1[1] * s1[2] + s1[0] * s1[1] * t1[2];
                    double vsum = 0.0;
                    for (int c = 0; c < ncent; c++) {
                        const double *C = cpos + 3 * c;
                        hermite_R(la + lb, p, P[0] - C[0], P[1] - C[1], P[2] - C[2], Rbuf);
                        double acc = 0.0;
                        int ix = ca[ia][0], jx = cb[ib][0], iy = ca[ia][1], jy = cb[ib][1];
                        int iz = ca[ia][2], jz = cb[ib][2];
                        for (int t = 0; t <= ix + jx; t++)
                            for (int u = 0; u <= iy + jy; u++)
                                for (int v = 0; v <= iz + jz; v++)
                                    acc += E[0][ix][jx][t] * E[1][iy][jy][u] * E[2][iz][jz][v] *
                                           Rbuf[(t * (MAXN + 1) + u) * (MAXN + 1) + v];
                        vsum -= charges[c] * acc;
                    }
                    V[row * n + col] = vsum * 2.0 * M_PI / p;
                }
        }
    free(off);
}

/* electric dipole integrals <a| r_d - origin_d |b>, d = x, y, z, over primitive Cartesian functions:
 * per direction (E^{ij}_1 + (P_d - O_d) E^{ij}_0) sqrt(pi/p), times the overlaps of the other two */
void dipole(int nsh, const int *l, const double *alpha, const double *ctr, const double *origin,
            double *Mx, double *My, double *Mz) {
    int n;
    int *off = shell_offsets(nsh, l, &n);
    double *M[3] = {Mx, My, Mz};
    for (int sa = 0; sa < nsh; sa++)
        for (int sb = 0; sb < nsh; sb++) {
            int la = l[sa], lb = l[sb];
            double a = alpha[sa], b = alpha[sb], p = a + b;
            const double *A = ctr + 3 * sa, *B = ctr + 3 * sb;
            double E[3][MAXL + 1][EJ][ET];
            for (int d = 0; d < 3; d++) hermite_E(la, lb, a, b, A[d], B[d], E[d]);
            int ca[6][3], cb[6][3];
            cart_components(la, ca);
            cart_components(lb, cb);
            double sq = sqrt(M_PI / p);
            for (int ia = 0; ia < ncart(la); ia++)
                for (int ib = 0; ib < ncart(lb); ib++) {
                    double s1[3], m1[3];
                    for (int d = 0; d < 3; d++) {
                        int i = ca[ia][d], j = cb[ib][d];
                        double P = (a * A[d] + b * B[d]) / p;
                        s1[d] = E[d][i][j][0] * sq;
                        m1[d] = (E[d][i][j][1] + (P - origin[d]) * E[d][i][j][0]) * sq;
                    }
                    int row = off[sa] + ia, col = off[sb] + ib;
                    M[0][row * n + col] = m1[0] * s1[1] * s1[2];
                    M[1][row * n + col] = s1[0] * m1[1] * s1[2];
                    M[2][row * n + col] = s1[0] * s1[1] * m1[2];
                }
        }
    free(off);
}

/* (ab|cd) over all primitive Cartesian functions, dense n^4 output */
void eri_all(int nsh, const int *l, const double *alpha, const double *ctr, double *out) {
    int n;
    int *off = shell_offsets(nsh, l, &n);
    static double Rbuf[(MAXN + 1) * (MAXN + 1) * (MAXN + 1)];
    for (int sa = 0; sa < nsh; sa++)
        for (int sb = 0; sb <= sa; sb++)
            for (int sc = 0; sc < nsh; sc++)
                for (int sd = 0; sd <= sc; sd++) {
                    if (sa * (sa + 1) / 2 + sb < sc * (sc + 1) / 2 + sd) continue;
                    int la = l[sa], lb = l[sb], lc = l[sc], ld = l[sd];
                    double a = alpha[sa], b = alpha[sb], c = alpha[sc], d = alpha[sd];
                    double p = a + b, q = c + d, al = p * q / (p + q);
                    const double *A = ctr + 3 * sa, *B = ctr + 3 * sb, *C = ctr + 3 * sc, *D = ctr + 3 * sd;
                    double Eab[3][MAXL + 1][EJ][ET], Ecd[3][MAXL + 1][EJ][ET];
                    double P[3], Q[3];
                    for (int k = 0; k < 3; k++) {
                        hermite_E(la, lb, a, b, A[k], B[k], Eab[k]);
                        hermite_E(lc, ld, c, d, C[k], D[k], Ecd[k]);
                        P[k] = (a * A[k] + b * B[k]) / p;
                        Q[k] = (c * C[k] + d * D[k]) / q;
                    }
                    int L = la + lb + lc + ld;
                    hermite_R(L, al, P[0] - Q[0], P[1] - Q[1], P[2] - Q[2], Rbuf);
                    double pref = 2.0 * pow(M_PI, 2.5) / (p * q * sqrt(p + q));
                    int ca[6][3], cb[6][3], cc[6][3], cd[6][3];
                    cart_components(la, ca);
                    cart_components(lb, cb);
                    cart_components(lc, cc);
                    cart_components(ld, cd);
                    for (int ia = 0; ia < ncart(la); ia++)
                        for (int ib = 0; ib < ncart(lb); ib++)
                            for (int ic = 0; ic < ncart(lc); ic++)
                                for (int id = 0; id < ncart(ld); id++) {
                                    int ax = ca[ia][0] , bx = cb[ib][0], cx = cc[ic][0], dx = cd[id][0];
                                    int ay = ca[ia][1] , by = cb[ib][1], cy = cc[ic][1], dy = cd[id][1];
                                    int az = ca[ia][2] , bz = cb[ib][2], cz = cc[ic][2], dz = cd[id][2];
                                    double acc = 0.0;
                                    for (int t = 0; t <= ax + bx; t++)
                                        for (int u = 0; u <= ay + by; u++)
                                            for (int v = 0; v <= az + bz; v++) {
                                                double e1 = Eab[0][ax][bx][t] * Eab[1][ay][by][u] * Eab[2][az][bz][v];
                                                if (e1 == 0.0) continue;
                                                double inner = 0.0;
                                                for (int tt = 0; tt <= cx + dx; tt++)
                                                    for (int uu = 0; uu <= cy + dy; uu++)
                                                        for (int vv = 0; vv <= cz + dz; vv++) {
                                                            double e2 = Ecd[0][cx][dx][tt] * Ecd[1][cy][dy][uu] *
                                                                        Ecd[2][cz][dz][vv];
                                                            double sgn = ((tt + uu + vv) & 1) ? -1.0 : 1.0;
                                                            inner += sgn * e2 *
                                                                     Rbuf[((t + tt) * (MAXN + 1) + (u + uu)) * (MAXN + 1) +
                                                                          (v + vv)];
                                                        }
                                                acc += e1 * inner;
                                            }
                                    double val = pref * acc;
                                    int i = off[sa] + ia, j = off[sb] + ib, k = off[sc] + ic, m = off[sd] + id;
                                    long n2 = (long)n * n, n3 = n2 * n;
                                    out[i * n3 + j * n2 + k * n + m] = val;
                                    out[j * n3 + i * n2 + k * n + m] = val;
                                    out[i * n3 + j * n2 + m * n + k] = val;
                                    out[j * n3 + i * n2 + m * n + k] = val;
                                    out[k * n3 + m * n2 + i * n + j] = val;
                                    out[m * n3 + k * n2 + i * n + j] = val;
                                    out[k * n3 + m * n2 + j * n + i] = val;
                                    out[m * n3 + k * n2 + j * n + i] = val;
                                }
                }
    free(off);
}
