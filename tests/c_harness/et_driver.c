/*
 * A C caller of libccsd_gpu.so that makes the calls eT's Fortran shim makes through its
 * ISO_C_BINDING interface block: column-major host arrays owned by the caller, int64 dimensions,
 * value scalars, int status codes, the Cholesky vectors in eT's four o/v blocks (J, p, q).
 *
 *   et_driver <input> <output>
 *
 * input  (native doubles / int64): n_o, n_v, n_J; L_oo, L_ov, L_vo, L_vv; h (n_mo^2); eps (n_mo);
 *        e_hf; t (n_amp); c (n_amp)
 * output: E; Omega (n_amp); rho = A c (n_amp); sigma = c^T A (n_amp)
 *
 * The sequence is eT's: wavefunction set-up, set_amplitudes (T1 transformation and Fock),
 * calculate_energy, construct_omega, prepare_for_jacobian, jacobian_transformation, then the
 * transpose on the same preparation.  Exit status 0 on success, 2 on a bad file, 3 on a library
 * status (printed with ccsd_gpu_last_error).
 */
#include <stdio.h>
#include <stdlib.h>

#include "ccsd_gpu.h"

static double *read_doubles(FILE *f, int64_t n) {
    double *p = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    if (p && fread(p, sizeof(double), (size_t)n, f) != (size_t)n) {
        free(p);
        return NULL;
    }
    return p;
}

static int failed(void *ctx, int rc, const char *what) {
    if (rc != CCSD_GPU_OK) {
        fprintf(stderr, "%s: status %d: %s\n", what, rc, ccsd_gpu_last_error(ctx));
        return 1;
    }
    return 0;
}

int main(int argc, char **argv) {
    if (argc != 3) {
        fprintf(stderr, "usage: %s <input> <output>\n", argv[0]);
        return 2;
    }
    FILE *in = fopen(argv[1], "rb");
    if (!in) return 2;
    int64_t dims[3];
    if (fread(dims, sizeof(int64_t), 3, in) != 3) return 2;
    const int64_t no = dims[0], nv = dims[1], nJ = dims[2], nmo = no + nv, nov = no * nv;
    const int64_t namp = nov + nov * (nov + 1) / 2;
    double *L_oo = read_doubles(in, nJ * no * no), *L_ov = read_doubles(in, nJ * no * nv);
    double *L_vo = read_doubles(in, nJ * nv * no), *L_vv = read_doubles(in, nJ * nv * nv);
    double *h = read_doubles(in, nmo * nmo), *eps = read_doubles(in, nmo), *e_hf = read_doubles(in, 1);
    double *t = read_doubles(in, namp), *c = read_doubles(in, namp);
    fclose(in);
    if (!L_oo || !L_ov || !L_vo || !L_vv || !h || !eps || !e_hf || !t || !c) return 2;
    double *omega = (double *)malloc(sizeof(double) * namp), *rho = (double *)malloc(sizeof(double) * namp);
    double *sigma = (double *)malloc(sizeof(double) * namp);
    double energy = 0.0;

    ccsd_gpu_options opt = {0};
    opt.device = 0;
    opt.precision = CCSD_GPU_FP64;
    void *ctx = NULL;
    if (failed(NULL, ccsd_gpu_create(no, nv, nJ, &opt, &ctx), "ccsd_gpu_create")) return 3;
    int bad = failed(ctx, ccsd_gpu_set_cholesky_mo_blocks(ctx, L_oo, L_ov, L_vo, L_vv), "set_cholesky_mo_blocks") ||
              failed(ctx, ccsd_gpu_set_h_mo(ctx, h, eps, *e_hf), "set_h_mo") ||
              failed(ctx, ccsd_gpu_set_amplitudes(ctx, t), "set_amplitudes") ||
              failed(ctx, ccsd_gpu_energy(ctx, &energy), "calculate_energy") ||
              failed(ctx, ccsd_gpu_omega(ctx, omega), "construct_omega") ||
              failed(ctx, ccsd_gpu_prepare_jacobian(ctx, 0), "prepare_for_jacobian") ||
              failed(ctx, ccsd_gpu_jacobian(ctx, 1, c, rho), "jacobian_transformation") ||
              failed(ctx, ccsd_gpu_prepare_jacobian(ctx, 1), "prepare_for_jacobian_transpose") ||
              failed(ctx, ccsd_gpu_jacobian_transpose(ctx, 1, c, sigma), "jacobian_transpose_transformation");
    ccsd_gpu_destroy(ctx);
    if (bad) return 3;

    FILE *out = fopen(argv[2], "wb");
    if (!out) return 2;
    fwrite(&energy, sizeof(double), 1, out);
    fwrite(omega, sizeof(double), (size_t)namp, out);
    fwrite(rho, sizeof(double), (size_t)namp, out);
    fwrite(sigma, sizeof(double), (size_t)namp, out);
    fclose(out);
    free(L_oo), free(L_ov), free(L_vo), free(L_vv), free(h), free(eps), free(e_hf), free(t), free(c);
    free(omega), free(rho), free(sigma);
    return 0;
}
