// Bandwidth kernels of the CCSD path: packed index algebra, A2 ladder +/- forms,
// energy, MP2 guess, quasi-Newton update and DIIS (all FP64).
#include <algorithm>
#include <cmath>

#include <cuda_bf16.h>

#include "ccsd_kernels.cuh"

namespace ccsd {

namespace {

__device__ __forceinline__ int64_t pk(int64_t x, int64_t y) {
    int64_t M = x > y ? x : y, m = x > y ? y : x;
    return M * (M + 1) / 2 + m;
}

// (M, m) with M >= m from a lower-triangle index M(M+1)/2 + m
__device__ __forceinline__ void untri(int64_t idx, int64_t &M, int64_t &m) {
    int64_t r = (int64_t)((sqrt(8.0 * (double)idx + 1.0) - 1.0) * 0.5);
    while (r * (r + 1) / 2 > idx) r--;
    while ((r + 1) * (r + 2) / 2 <= idx) r++;
    M = r;
    m = idx - r * (r + 1) / 2;
}

inline int grid_for(int64_t total, int block) {
    int64_t g = (total + block - 1) / block;
    if (g < 1) g = 1;
    if (g > 148 * 64) g = 148 * 64;
    return (int)g;
}

#define GRID_STRIDE(i, total) \
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (total); i += (int64_t)gridDim.x * blockDim.x)

__global__ void build_tpm_kernel(const double *__restrict__ t2, double *__restrict__ tp, double *__restrict__ tm,
                                 int64_t no, int64_t nv, int64_t ldp, int64_t ldm) {
    const int64_t nop = no * (no + 1) / 2, nvp = nv * (nv + 1) / 2;
    GRID_STRIDE(idx, nop * nvp) {
        int64_t ij = idx % nop, cd = idx / nop, i, j, c, d;
        untri(ij, i, j);
        untri(cd, c, d);
        double a = t2[pk(c + nv * i, d + nv * j)];
        double b = t2[pk(c + nv * j, d + nv * i)];
        double f = (c == d ? 0.5 : 1.0) * (i == j ? 0.5 : 1.0);
        tp[ij + ldp * cd] = f * (a + b);
        if (i > j && c > d) {
            int64_t ijm = i * (i - 1) / 2 + j, cdm = c * (c - 1) / 2 + d;
            tm[ijm + ldm * cdm] = a - b;
        }
    }
}

// G[(c + nv*(a-a0)) + ldg*(d + nv*b)] = g_acbd for a in [a0,a1), b in [0,a1)
__global__ void form_gpm_kernel(const double *__restrict__ G, int64_t ldg, double *__restrict__ gp,
                                double *__restrict__ gm, int64_t nv, int64_t a0, int64_t a1) {
    const int64_t nvp = nv * (nv + 1) / 2, nvm = nv * (nv - 1) / 2;
    const int64_t abp0 = a0 * (a0 + 1) / 2, nabp = a1 * (a1 + 1) / 2 - abp0;
    const int64_t abm0 = a0 * (a0 - 1) / 2;
    GRID_STRIDE(idx, nvp * nabp) {
        int64_t cd = idx % nvp, loc = idx / nvp, a, b, c, d;
        untri(abp0 + loc, a, b);
        untri(cd, c, d);
        double x = G[(c + nv * (a - a0)) + ldg * (d + nv * b)];
        double y = G[(d + nv * (a - a0)) + ldg * (c + nv * b)];
        gp[idx] = x + y;
        if (a > b && c > d) {
            int64_t cdm = c * (c - 1) / 2 + d, locm = a * (a - 1) / 2 + b - abm0;
            gm[cdm + nvm * locm] = x - y;
        }
    }
}

// bf16 rounding planes of x: plane q holds the rounding of x minus the planes before it
__device__ __forceinline__ void put_planes(double x, int np, size_t plane, __nv_bfloat16 *out) {
    for (int q = 0; q < np; q++) {
        const __nv_bfloat16 h = __double2bfloat16(x);
        out[q * plane] = h;
        x -= (double)__bfloat162float(h);
    }
}

// t+ (plus) or t- rows of the +/- tensor-core ladder as np bf16 planes [np][rows_pad][kpad]: row
// vec n_rows + ij (vector vec, ij over i >= j for t+, i > j for t-), column cd over c >= d (t+) or
// c > d (t-), the values of build_tpm
__global__ void build_tpm_planes_kernel(const double *__restrict__ t2s, int64_t nvec, int64_t no, int64_t nv,
                                        int64_t rows_pad, int64_t kpad, int np, int plus,
                                        __nv_bfloat16 *__restrict__ out) {
    const int64_t nrow = plus ? no * (no + 1) / 2 : no * (no - 1) / 2;
    const int64_t ncol = plus ? nv * (nv + 1) / 2 : nv * (nv - 1) / 2;
    const int64_t nt2 = nv * no * (nv * no + 1) / 2;
    const size_t plane = (size_t)rows_pad * kpad;
    GRID_STRIDE(idx, rows_pad * kpad) {
        const int64_t rr = idx / kpad, k = idx - rr * kpad;
        const int64_t vec = nrow > 0 ? rr / nrow : nvec, row = nrow > 0 ? rr - vec * nrow : 0;
        double val = 0.0;
        if (vec < nvec && k < ncol) {
            int64_t i, j, c, d;
            untri(row, i, j);
            untri(k, c, d);
            if (!plus) {   // strict triangles: M(M-1)/2 + m maps to (M-1, m)
                i += 1;
                c += 1;
            }
            const double *t2 = t2s + vec * nt2;
            const double x = t2[pk(c + nv * i, d + nv * j)], y = t2[pk(c + nv * j, d + nv * i)];
            val = plus ? (c == d ? 0.5 : 1.0) * (i == j ? 0.5 : 1.0) * (x + y) : x - y;
        }
        put_planes(val, np, plane, out + idx);
    }
}

// g+- of one block of a from G[(c + nv (a - a0)) + ldg (d + nv b)] = g_acbd (a in [a0, a1), b <= a):
// g+ = g_acbd + g_adbc (c >= d) into P+ row a(a+1)/2 + b - rowp0, column c(c+1)/2 + d; g- = g_acbd -
// g_adbc (a > b, c > d) into P- row a(a-1)/2 + b - rowm0, column c(c-1)/2 + d; each as np bf16
// planes.  A block of threads takes one pair (a, b) and one 32 x 32 tile of (c, d) with its mirror
// tile, staged in shared memory so that both reads run along c and the writes along d.
__global__ void form_pm_planes_kernel(const double *__restrict__ G, int64_t ldg, int64_t nv, int64_t a0, int64_t a1,
                                      int np, __nv_bfloat16 *__restrict__ Pp, int64_t kp, size_t plane_p,
                                      int64_t rowp0, __nv_bfloat16 *__restrict__ Pm, int64_t km, size_t plane_m,
                                      int64_t rowm0) {
    __shared__ double sA[32][33], sB[32][33];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int64_t abp0 = a0 * (a0 + 1) / 2, npairs = a1 * (a1 + 1) / 2 - abp0;
    int64_t ct, dt;
    untri(blockIdx.x, ct, dt);                       // tile pair ct >= dt
    const int64_t c0 = 32 * ct, d0 = 32 * dt;
    for (int64_t loc = blockIdx.y; loc < npairs; loc += gridDim.y) {
        int64_t a, b;
        untri(abp0 + loc, a, b);
        const double *Gab = G + nv * (a - a0) + ldg * nv * b;   // Gab[c + ldg d] = g_acbd
        for (int j = ty; j < 32; j += 8) {
            const int64_t c = c0 + tx, d = d0 + j, cm = d0 + tx, dm = c0 + j;
            sA[j][tx] = (c < nv && d < nv) ? Gab[c + ldg * d] : 0.0;       // g_acbd, c = c0 + tx
            sB[j][tx] = (cm < nv && dm < nv) ? Gab[cm + ldg * dm] : 0.0;   // g_a(d0+tx)b(c0+j)
        }
        __syncthreads();
        const int64_t d = d0 + tx;
        for (int i = ty; i < 32; i += 8) {
            const int64_t c = c0 + i;
            if (c < nv && d <= c) {
                const double x = sA[tx][i], y = sB[i][tx];      // g_acbd, g_adbc
                put_planes(x + y, np, plane_p, Pp + (a * (a + 1) / 2 + b - rowp0) * kp + c * (c + 1) / 2 + d);
                if (a > b && d < c)
                    put_planes(x - y, np, plane_m, Pm + (a * (a - 1) / 2 + b - rowm0) * km + c * (c - 1) / 2 + d);
            }
        }
        __syncthreads();
    }
}

__global__ void add_omega_pm_kernel(double *__restrict__ om2, const double *__restrict__ wp,
                                    const double *__restrict__ wm, int64_t no, int64_t nv, int64_t a0, int64_t a1,
                                    int64_t ldwp, int64_t ldwm) {
    const int64_t nop = no * (no + 1) / 2;
    const int64_t abp0 = a0 * (a0 + 1) / 2, nabp = a1 * (a1 + 1) / 2 - abp0;
    const int64_t abm0 = a0 * (a0 - 1) / 2;
    GRID_STRIDE(idx, nop * nabp) {
        int64_t ij = idx % nop, loc = idx / nop, i, j, a, b;
        untri(ij, i, j);
        untri(abp0 + loc, a, b);
        double p = wp[ij + ldwp * loc] * (a == b ? 0.5 : 1.0);
        double x1 = p, x2 = p;
        if (i != j && a != b) {
            int64_t ijm = i * (i - 1) / 2 + j, locm = a * (a - 1) / 2 + b - abm0;
            double m = wm[ijm + ldwm * locm];
            x1 = p + m;
            x2 = p - m;
        }
        int64_t P1 = pk(a + nv * i, b + nv * j), P2 = pk(a + nv * j, b + nv * i);
        if (P1 == P2) {
            om2[P1] += x1 + x2;
        } else {
            om2[P1] += x1;
            om2[P2] += x2;
        }
    }
}

// D += the h-derivative of the energy at fixed amplitudes: 2 on the occupied diagonal (reference)
// and 2 t_ai at (i, n_o + a) (the singles term through h~_ii = h_ii + sum_a h_ia t_ai)
__global__ void density_energy_part_kernel(double *__restrict__ D, const double *__restrict__ t1, int64_t no,
                                           int64_t nv) {
    const int64_t nmo = no + nv;
    GRID_STRIDE(idx, no * nv + no) {
        if (idx < no) {
            D[idx + nmo * idx] += 2.0;
        } else {
            const int64_t k = idx - no, a = k % nv, i = k / nv;   // t1 (v, o): t_ai at a + nv i
            D[i + nmo * (no + a)] += 2.0 * t1[a + nv * i];
        }
    }
}

// eta_ai = 2 F_ia, eta_aibj = 4 g_iajb - 2 g_ibja packed (construct_eta_ccsd); F is n_mo x n_mo,
// g is (o, v, o, v)
__global__ void eta_kernel(const double *__restrict__ F, const double *__restrict__ g, int64_t no, int64_t nv,
                           double *__restrict__ eta) {
    const int64_t nov = no * nv, nt2 = nov * (nov + 1) / 2, nmo = no + nv;
    GRID_STRIDE(k, nov + nt2) {
        if (k < nov) {
            int64_t a = k % nv, i = k / nv;
            eta[k] = 2.0 * F[i + nmo * (no + a)];
        } else {
            int64_t M, m;
            untri(k - nov, M, m);
            int64_t a = M % nv, i = M / nv, b = m % nv, j = m / nv;
            eta[k] = 4.0 * g[i + no * (a + nv * (j + no * b))] - 2.0 * g[i + no * (b + nv * (j + no * a))];
        }
    }
}

// t1bar = t1, t2bar = 2 t_aibj - t_ajbi (packed contravariant amplitudes)
__global__ void multiplier_guess_kernel(const double *__restrict__ t, int64_t no, int64_t nv,
                                        double *__restrict__ out) {
    const int64_t nov = no * nv, nt2 = nov * (nov + 1) / 2;
    GRID_STRIDE(k, nov + nt2) {
        if (k < nov) out[k] = t[k];
        else {
            int64_t M, m;
            untri(k - nov, M, m);
            int64_t a = M % nv, i = M / nv, b = m % nv, j = m / nv;
            out[k] = 2.0 * t[nov + k - nov] - t[nov + pk(a + nv * j, b + nv * i)];
        }
    }
}

// E_corr partial sums: sum_{ai,bj} (t_aibj + t_ai t_bj)(2 g_iajb - g_ibja), g (o,v,o,v)
__global__ void energy_partial_kernel(const double *__restrict__ t1, const double *__restrict__ t2,
                                      const double *__restrict__ g, int64_t no, int64_t nv,
                                      double *__restrict__ partial) {
    const int64_t nov = no * nv;
    double acc = 0.0;
    GRID_STRIDE(idx, nov * nov) {
        int64_t ai = idx % nov, bj = idx / nov;
        int64_t a = ai % nv, i = ai / nv, b = bj % nv, j = bj / nv;
        double t = t2[pk(ai, bj)] + t1[ai] * t1[bj];
        double g1 = g[i + no * (a + nv * (j + no * b))];
        double g2 = g[i + no * (b + nv * (j + no * a))];
        acc += t * (2.0 * g1 - g2);
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    __shared__ double sh[32];
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double r = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
        if (threadIdx.x == 0) partial[blockIdx.x] = r;
    }
}

// E_corr partial sums from the packed doubles: the (ia, jb) matrix of g_iajb is symmetric
// (g_iajb = g_jbia), so its o x o sub-block P_ab[i,j] = g_iajb also gives g_ibja = P_ab[j,i] and
// serves both orders of the virtual pair:
//   E_ab + E_ba = sum_ij T[ai,bj] (2 P[i,j] - P[j,i]) + T[bi,aj] (2 P[j,i] - P[i,j]),
// T = t2 + t1 t1.  One pair a >= b at a time per block: P is staged in shared memory (read once,
// coalesced along i), and every packed t2 element belongs to exactly one pair, so the kernel reads
// half of g and all of t2 once.  Pairs run in packed order (b fastest), so blocks resident together
// share the DRAM sectors of neighbouring t2 rows.
__global__ void energy_pairs_kernel(const double *__restrict__ t1, const double *__restrict__ t2,
                                    const double *__restrict__ g, int no, int64_t nv, int64_t npairs,
                                    double *__restrict__ partial) {
    extern __shared__ double P[];   // (no + 1) x no, padded against bank conflicts
    const int ld = no + 1, nn = no * no;
    double acc = 0.0;
    for (int64_t p = blockIdx.x; p < npairs; p += gridDim.x) {
        int64_t a, b;
        untri(p, a, b);
        __syncthreads();
        for (int k = threadIdx.x; k < nn; k += blockDim.x) {
            const int i = k % no, j = k / no;
            P[i + ld * j] = g[i + no * (a + nv * (j + (int64_t)no * b))];
        }
        __syncthreads();
        for (int k = threadIdx.x; k < nn; k += blockDim.x) {
            const int i = k % no, j = k / no;
            const double pij = P[i + ld * j], pji = P[j + ld * i];
            const int64_t ai = a + nv * i, bj = b + nv * j;
            acc += (t2[pk(ai, bj)] + t1[ai] * t1[bj]) * (2.0 * pij - pji);
            if (a != b) {
                const int64_t bi = b + nv * i, aj = a + nv * j;
                acc += (t2[pk(bi, aj)] + t1[bi] * t1[aj]) * (2.0 * pji - pij);
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    __shared__ double sh[32];
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double r = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
        if (threadIdx.x == 0) partial[blockIdx.x] = r;
    }
}

__global__ void sum_partial_kernel(const double *__restrict__ partial, int n, double add, double *__restrict__ out) {
    __shared__ double sh[32];
    double acc = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) acc += partial[i];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double r = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
        if (threadIdx.x == 0) out[0] = r + add;
    }
}

__global__ void orbital_differences_kernel(const double *__restrict__ eps, int64_t no, int64_t nv,
                                           double *__restrict__ out) {
    const int64_t nov = no * nv, nt2 = nov * (nov + 1) / 2;
    GRID_STRIDE(k, nov + nt2) {
        if (k < nov) {
            int64_t a = k % nv, i = k / nv;
            out[k] = eps[no + a] - eps[i];
        } else {
            int64_t M, m;
            untri(k - nov, M, m);
            int64_t a = M % nv, i = M / nv, b = m % nv, j = m / nv;
            out[k] = eps[no + a] - eps[i] + eps[no + b] - eps[j];
        }
    }
}

// t2 = g_aibj / (e_i + e_j - e_a - e_b) with g (v,o,v,o) = sum_J L_ai L_bj
__global__ void mp2_kernel(const double *__restrict__ g, const double *__restrict__ epsdiff, int64_t nov,
                           double *__restrict__ t2) {
    const int64_t nt2 = nov * (nov + 1) / 2;
    GRID_STRIDE(k, nt2) {
        int64_t M, m;
        untri(k, M, m);
        t2[k] = -g[m + nov * M] / epsdiff[nov + k];
    }
}

// trace X_J = sum_k L[J,k,k] over an (nJ, no, no) block
__global__ void trace_kernel(const double *__restrict__ L, int64_t nJ, int64_t no, double *__restrict__ X) {
    GRID_STRIDE(J, nJ) {
        double s = 0.0;
        for (int64_t k = 0; k < no; k++) s += L[J + nJ * (k + no * k)];
        X[J] = s;
    }
}

__device__ __forceinline__ bool is_doubles_diag(int64_t k, int64_t nt1) {
    if (k < nt1) return false;
    int64_t M, m;
    untri(k - nt1, M, m);
    return M == m;
}

// residual <- -omega/eps; update = residual (doubles diagonal x2); t += update; residual diagonal x2
__global__ void qn_update_kernel(double *__restrict__ omega, const double *__restrict__ epsdiff,
                                 double *__restrict__ t, int64_t n, int64_t nt1) {
    GRID_STRIDE(k, n) {
        double r = -omega[k] / epsdiff[k];
        if (is_doubles_diag(k, nt1)) r *= 2.0;
        t[k] += r;
        omega[k] = r;
    }
}

// the quasi-Newton image of a residual without the amplitude update: v <- -v / eps, doubles
// diagonal x2 (the DIIS error vector of quasi_newton_updater_class.F90)
__global__ void qn_precondition_kernel(double *__restrict__ v, const double *__restrict__ epsdiff, int64_t n,
                                       int64_t nt1) {
    GRID_STRIDE(k, n) {
        double r = -v[k] / epsdiff[k];
        if (is_doubles_diag(k, nt1)) r *= 2.0;
        v[k] = r;
    }
}

__global__ void scale_doubles_diag_kernel(double *__restrict__ x, int64_t nov, int64_t nt1, double f) {
    GRID_STRIDE(M, nov) {
        x[nt1 + M * (M + 1) / 2 + M] *= f;
    }
}

struct Ptr16 {
    const double *p[16];
    double w[16];
};

// x = sum_k w_k p_k  (weights read from device memory)
__global__ void extrapolate_kernel(Ptr16 recs, const double *__restrict__ w, int nrec, int64_t n,
                                   double *__restrict__ x) {
    GRID_STRIDE(i, n) {
        double s = 0.0;
        for (int k = 0; k < nrec; k++) s += w[k] * recs.p[k][i];
        x[i] = s;
    }
}

// Insert the new dot products into the slot-indexed Gram matrix, build the padded DIIS
// system in logical (oldest -> newest) order and solve it by Gaussian elimination with
// partial pivoting (dgesv semantics).  Writes w[slot]; status[0] = 0 ok / 1 singular.
__global__ void diis_solve_kernel(double *__restrict__ Gslot, int maxdim, const double *__restrict__ dots,
                                  int new_slot, DiisOrder order, double *__restrict__ w, int *__restrict__ status) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int n = order.n;
    for (int k = 0; k < n; k++) {
        int s = order.slot[k];
        Gslot[new_slot * maxdim + s] = dots[s];
        Gslot[s * maxdim + new_slot] = dots[s];
    }
    double A[17][18];
    const int m = n + 1;
    for (int r = 0; r < n; r++) {
        for (int c = 0; c < n; c++) A[r][c] = Gslot[order.slot[r] * maxdim + order.slot[c]];
        A[r][n] = -1.0;
        A[r][m] = 0.0;
    }
    for (int c = 0; c < n; c++) A[n][c] = -1.0;
    A[n][n] = 0.0;
    A[n][m] = -1.0;
    int st = 0;
    for (int col = 0; col < m; col++) {
        int piv = col;
        double best = fabs(A[col][col]);
        for (int r = col + 1; r < m; r++)
            if (fabs(A[r][col]) > best) {
                best = fabs(A[r][col]);
                piv = r;
            }
        if (best == 0.0) {
            st = 1;
            break;
        }
        if (piv != col)
            for (int c = 0; c <= m; c++) {
                double tmp = A[col][c];
                A[col][c] = A[piv][c];
                A[piv][c] = tmp;
            }
        for (int r = col + 1; r < m; r++) {
            double f = A[r][col] / A[col][col];
            for (int c = col; c <= m; c++) A[r][c] -= f * A[col][c];
        }
    }
    double x[17];
    if (!st) {
        for (int r = m - 1; r >= 0; r--) {
            double s = A[r][m];
            for (int c = r + 1; c < m; c++) s -= A[r][c] * x[c];
            x[r] = s / A[r][r];
        }
        for (int k = 0; k < n; k++) w[k] = x[k];
    }
    status[0] = st;
}

}  // namespace

void build_tpm(Exec &ex, const double *t2, double *tp, double *tm, int64_t no, int64_t nv, int64_t ldp, int64_t ldm) {
    int64_t total = (no * (no + 1) / 2) * (nv * (nv + 1) / 2);
    build_tpm_kernel<<<grid_for(total, 256), 256, 0, ex.stream>>>(t2, tp, tm, no, nv, ldp, ldm);
    ex.launches++;
    CU_CHECK(cudaGetLastError());
}

void form_gpm(Exec &ex, const double *G, int64_t ldg, double *gp, double *gm, int64_t nv, int64_t a0, int64_t a1) {
    int64_t total = (nv * (nv + 1) / 2) * (a1 * (a1 + 1) / 2 - a0 * (a0 + 1) / 2);
    form_gpm_kernel<<<grid_for(total, 256), 256, 0, ex.stream>>>(G, ldg, gp, gm, nv, a0, a1);
    ex.launches++;
    CU_CHECK(cudaGetLastError());
}

void add_omega_pm(Exec &ex, double *om2, const double *wp, const double *wm, int64_t no, int64_t nv, int64_t a0,
                  int64_t a1, int64_t ldwp, int64_t ldwm) {
    int64_t total = (no * (no + 1) / 2) * (a1 * (a1 + 1) / 2 - a0 * (a0 + 1) / 2);
    add_omega_pm_kernel<<<grid_for(total, 256), 256, 0, ex.stream>>>(om2, wp, wm, no, nv, a0, a1, ldwp, ldwm);
    ex.launches++;
    CU_CHECK(cudaGetLastError());
}

void build_tpm_planes(Exec &ex, const double *t2s, int64_t nvec, int64_t no, int64_t nv, bool plus, int64_t rows_pad,
                      int64_t kpad, int np, __nv_bfloat16 *out) {
    build_tpm_planes_kernel<<<grid_for(rows_pad * kpad, 256), 256, 0, ex.stream>>>(t2s, nvec, no, nv, rows_pad, kpad,
                                                                                  np, plus ? 1 : 0, out);
    ex.launches++;
    CU_CHECK(cudaGetLastError());
}

void form_pm_planes(Exec &ex, const double *G, int64_t ldg, int64_t nv, int64_t a0, int64_t a1, int np,
                    __nv_bfloat16 *Pp, int64_t kp, size_t plane_p, int64_t rowp0, __nv_bfloat16 *Pm, int64_t km,
                    size_t plane_m, int64_t rowm0) {
    const int64_t nt = (nv + 31) / 32, npairs = a1 * (a1 + 1) / 2 - a0 * (a0 + 1) / 2;
    dim3 grid((unsigned)(nt * (nt + 1) / 2), (unsigned)std::min<int64_t>(npairs, 65535));
    form_pm_planes_kernel<<<grid, dim3(32, 8), 0, ex.stream>>>(G, ldg, nv, a0, a1, np, Pp, kp, plane_p, rowp0, Pm, km,
                                                              plane_m, rowm0);
    ex.launches++;
    CU_CHECK(cudaGetLastError());
}

void density_energy_part(Exec &ex, double *D, const double *t1, int64_t no, int64_t nv) {
    density_energy_part_kernel<<<grid_for(no * nv + no, 256), 256, 0, ex.stream>>>(D, t1, no, nv);
    ex.launches++;
    CU_CHECK(cudaGetLastError());
}

void construct_eta(Exec &ex, const double *F, const double *g_ovov, int64_t no, int64_t nv, double *eta) {
    int64_t nov = no * nv, total = nov + nov * (nov + 1) / 2;
    eta_kernel<<<grid_for(total, 256), 256, 0, ex.stream>>>(F, g_ovov, no, nv, eta);
    ex.launches++;
    CU_CHECK(cudaGetLastError());
}

void multiplier_guess(Exec &ex, const double *t, int64_t no, int64_t nv, double *out) {
    int64_t nov = no * nv, total = nov + nov * (nov + 1) / 2;
    multiplier_guess_kernel<<<grid_for(total, 256), 256, 0, ex.stream>>>(t, no, nv, out);
    ex.launches++;
    CU_CHECK(cudaGetLastError());
}

void energy_reduce(Exec &ex, const double *t1, const double *t2, const double *g_ovov, int64_t no, int64_t nv,
                   double add, double *d_out) {
    const int nb = 592;
    DBuf part = dalloc(nb, ex.stream);
    if (no <= 64) {
        // staged sub-blocks of up to 64 x 65 doubles (33 KB of shared memory)
        const size_t smem = sizeof(double) * (size_t)(no + 1) * (size_t)no;
        energy_pairs_kernel<<<nb, 256, smem, ex.stream>>>(t1, t2, g_ovov, (int)no, nv, nv * (nv + 1) / 2, part.d());
    } else {
        energy_partial_kernel<<<nb, 256, 0, ex.stream>>>(t1, t2, g_ovov, no, nv, part.d());
    }
    sum_partial_kernel<<<1, 256, 0, ex.stream>>>(part.d(), nb, add, d_out);
    ex.launches += 2;
    CU_CHECK(cudaGetLastError());
}

void orbital_differences(Exec &ex, const double *eps, int64_t no, int64_t nv, double *out) {
    int64_t nov = no * nv, total = nov + nov * (nov + 1) / 2;
    orbital_differences_kernel<<<grid_for(total, 256), 256, 0, ex.stream>>>(eps, no, nv, out);
    ex.launches++;
    CU_CHECK(cudaGetLastError());
}

void mp2_amplitudes(Exec &ex, const double *g_vovo, const double *epsdiff, int64_t nov, double *t2) {
    mp2_kernel<<<grid_for(nov * (nov + 1) / 2, 256), 256, 0, ex.stream>>>(g_vovo, epsdiff, nov, t2);
    ex.launches++;
    CU_CHECK(cudaGetLastError());
}

void trace_oo(Exec &ex, const double *L_oo, int64_t nJ, int64_t no, double *X) {
    trace_kernel<<<grid_for(nJ, 128), 128, 0, ex.stream>>>(L_oo, nJ, no, X);
    ex.launches++;
    CU_CHECK(cudaGetLastError());
}

void qn_update(Exec &ex, double *omega, const double *epsdiff, double *t, int64_t n, int64_t nt1) {
    qn_update_kernel<<<grid_for(n, 256), 256, 0, ex.stream>>>(omega, epsdiff, t, n, nt1);
    ex.launches++;
    CU_CHECK(cudaGetLastError());
}

void qn_precondition(Exec &ex, double *v, const double *epsdiff, int64_t n, int64_t nt1) {
    qn_precondition_kernel<<<grid_for(n, 256), 256, 0, ex.stream>>>(v, epsdiff, n, nt1);
    ex.launches++;
    CU_CHECK(cudaGetLastError());
}

void scale_doubles_diag(Exec &ex, double *x, int64_t nov, int64_t nt1, double f) {
    scale_doubles_diag_kernel<<<grid_for(nov, 256), 256, 0, ex.stream>>>(x, nov, nt1, f);
    ex.launches++;
    CU_CHECK(cudaGetLastError());
}

void diis_solve(Exec &ex, double *Gslot, int maxdim, const double *dots, int new_slot, const DiisOrder &order,
                double *w, int *status) {
    diis_solve_kernel<<<1, 32, 0, ex.stream>>>(Gslot, maxdim, dots, new_slot, order, w, status);
    ex.launches++;
    CU_CHECK(cudaGetLastError());
}

void extrapolate(Exec &ex, const double *const *recs, const double *w, int nrec, int64_t n, double *x) {
    Ptr16 p{};
    for (int k = 0; k < nrec; k++) p.p[k] = recs[k];
    extrapolate_kernel<<<grid_for(n, 256), 256, 0, ex.stream>>>(p, w, nrec, n, x);
    ex.launches++;
    CU_CHECK(cudaGetLastError());
}

}  // namespace ccsd
