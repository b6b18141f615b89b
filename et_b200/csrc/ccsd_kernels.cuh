// Bandwidth kernels of the CCSD path (declarations).
#pragma once

#include <cuda_bf16.h>

#include "common.cuh"

namespace ccsd {

struct DiisOrder {
    int n;          // active records
    int slot[16];   // record slots, oldest first
};

// t+ (n_o_p x n_v_p) and t- (n_o_m x n_v_m) of the A2 ladder (construct_plus_minus_2413_from_packed
// followed by scale_double_packed_blocks(1/2, 1/2); packed_array_utilities_r.F90:140-197, 99-136)
// (tp leading dimension ldp >= n_o_p, tm leading dimension ldm >= n_o_m: several vectors side by side)
void build_tpm(Exec &ex, const double *t2, double *tp, double *tm, int64_t no, int64_t nv, int64_t ldp, int64_t ldm);
// g+- columns for the pairs a in [a0,a1), b <= a from G = g_acbd (construct_plus_minus_1324_from_full)
void form_gpm(Exec &ex, const double *G, int64_t ldg, double *gp, double *gm, int64_t nv, int64_t a0, int64_t a1);
// add_double/single_packed_plus_minus with the omega+ (a == b) half scaling
void add_omega_pm(Exec &ex, double *om2, const double *wp, const double *wm, int64_t no, int64_t nv, int64_t a0,
                  int64_t a1, int64_t ldwp, int64_t ldwm);

// the +/- ladder on the tensor cores: t+ (plus) or t- of nvec packed vectors as np bf16 planes
// [np][rows_pad][kpad] (rows: vector-major i >= j or i > j; columns: c >= d or c > d; build_tpm's
// values), and g+- of the pairs a in [a0, a1) as planes of P+ [np][.][kp] (rows a(a+1)/2 + b - rowp0)
// and P- [np][.][km] (rows a(a-1)/2 + b - rowm0) from G = g_acbd in form_gpm's layout
void build_tpm_planes(Exec &ex, const double *t2s, int64_t nvec, int64_t no, int64_t nv, bool plus, int64_t rows_pad,
                      int64_t kpad, int np, __nv_bfloat16 *out);
void form_pm_planes(Exec &ex, const double *G, int64_t ldg, int64_t nv, int64_t a0, int64_t a1, int np,
                    __nv_bfloat16 *Pp, int64_t kp, size_t plane_p, int64_t rowp0, __nv_bfloat16 *Pm, int64_t km,
                    size_t plane_m, int64_t rowm0);

// eta of the multiplier equation (construct_eta_ccsd, multiplier_equation_ccsd.F90:50-113) and the
// initial multipliers (t1, packed contravariant t2; ccsd_class.F90:411-475)
// D (n_mo x n_mo) += dE/dh at fixed amplitudes (reference 2 on the occupied diagonal, 2 t_ai at (i, a))
void density_energy_part(Exec &ex, double *D, const double *t1, int64_t no, int64_t nv);
void construct_eta(Exec &ex, const double *F, const double *g_ovov, int64_t no, int64_t nv, double *eta);
void multiplier_guess(Exec &ex, const double *t, int64_t no, int64_t nv, double *out);

void energy_reduce(Exec &ex, const double *t1, const double *t2, const double *g_ovov, int64_t no, int64_t nv,
                   double add, double *d_out);
void orbital_differences(Exec &ex, const double *eps, int64_t no, int64_t nv, double *out);
void mp2_amplitudes(Exec &ex, const double *g_vovo, const double *epsdiff, int64_t nov, double *t2);
void trace_oo(Exec &ex, const double *L_oo, int64_t nJ, int64_t no, double *X);
void qn_update(Exec &ex, double *omega, const double *epsdiff, double *t, int64_t n, int64_t nt1);
// v <- the quasi-Newton image of the residual v (-v / eps, doubles diagonal x2), t untouched
void qn_precondition(Exec &ex, double *v, const double *epsdiff, int64_t n, int64_t nt1);
void scale_doubles_diag(Exec &ex, double *x, int64_t nov, int64_t nt1, double f);
void diis_solve(Exec &ex, double *Gslot, int maxdim, const double *dots, int new_slot, const DiisOrder &order,
                double *w, int *status);
void extrapolate(Exec &ex, const double *const *recs, const double *w, int nrec, int64_t n, double *x);

}  // namespace ccsd
