// The per-system context behind the C ABI.
#pragma once

#include <string>

#include "common.cuh"

namespace ccsd {

struct Context {
    int64_t no, nv, nJ, nmo, nov, nt1, nt2, namp;
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cublasHandle_t blas = nullptr;
    Exec ex;
    GemmProfile prof;
    int64_t ladder_batch = 0;
    double e_hf = 0.0;
    bool have_L = false, have_h = false, have_t = false;
    std::string err;

    // MO Cholesky blocks (J, p, q) and their T1-transformed counterparts
    DBuf L_oo, L_ov, L_vo, L_vv;
    DBuf Lt_oo, Lt_ov, Lt_vo, Lt_vv;
    DBuf h, eps, F;          // h_mo, orbital energies, T1 Fock (n_mo x n_mo)
    DBuf t;                  // [t1 | packed t2]
    DBuf epsdiff;            // orbital differences (n_amp)
    DBuf scal;               // scalar scratch
    DBuf mbuf;               // split-bf16 ladder integrals M_ab[c,d] for all pairs (mixed precision)
    size_t mbuf_bytes = 0;

    Context(int64_t no, int64_t nv, int64_t nJ, const ccsd_gpu_options *opt);
    ~Context();

    void set_stream(cudaStream_t s);
    void t1_transform_cholesky();
    void construct_fock();
    void refresh();                        // T1 transformation + Fock at the current t
    DBuf g_ovov();
    double energy();
    void mp2_guess();
    void omega(double *d_omega);
    void ladder(const double *t2, double *om2);
    void ladder_tc(const double *t2, double *om2);
    int solve_gs(const ccsd_gpu_solver_options *o, double *energy, int32_t *iters, double *history);
    double omega_flops() const;
};

}  // namespace ccsd
