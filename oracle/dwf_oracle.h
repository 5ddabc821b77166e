/*
 * CPU oracle for the even-odd 5D domain-wall operator and its solvers.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * Bridge++ corelib algorithm (AFopr_Domainwall_eo<Field> over Fopr_Wilson_eo,
 * Solver_CG, AShiftsolver_CG).  It exists to check the CUDA product path; the
 * product never links, loads or calls it.
 *
 * Field layouts are the corelib host layouts:
 *   links (lexical)  : ri + 2*(col + 3*row) + 18*(site + Nvol*mu)
 *   5D half spinor   : ri + 2*(color + 3*spin) + 24*(site_eo + Nvol2*s)
 */
#ifndef DWF_ORACLE_H
#define DWF_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_dwf oracle_dwf;

oracle_dwf *oracle_dwf_create(const int lattice[4], int Ls, double mq,
                              double M0, const double *b, const double *c,
                              double alpha, const int bc[4]);
void oracle_dwf_destroy(oracle_dwf *op);

/* Lexical links -> even/odd links held by the oracle. */
void oracle_dwf_set_links(oracle_dwf *op, const double *u_lex);

/* Operator apply by reference mode name:
 *   Deo Doe Dee Doo Dee_inv Doo_inv D Ddag DdagD H Hdag gm5R R
 * dag != 0 selects mult_dag (e.g. dag+"Deo" = Ddag_eo(.,1), dag+"D" = Ddag).
 * Returns 0, or -1 for an unknown mode. */
int oracle_dwf_mult(oracle_dwf *op, const char *mode, int dag, double *out,
                    const double *in);

/* Conjugate gradient on DdagD (reference src/lib_alt/Solver/
 * asolver_CG-tmpl.h:118-234, zero initial guess).  Stops when
 * |r|^2/|b|^2 < tol2.  Returns 0 if converged. */
int oracle_cg(oracle_dwf *op, double *x, const double *b, double tol2,
              int maxiter, int *nconv, double *diff);

/* Multishift CG on DdagD + sigma_i (reference src/lib/Solver/
 * ashiftsolver_CG-tmpl.h:89-329).  x holds nshift consecutive fields. */
int oracle_shiftcg(oracle_dwf *op, double *x, const double *sigma, int nshift,
                   const double *b, double tol2, int maxiter, int *nconv,
                   double *diff);

/* Fermion force of Force_F_Domainwall_eo (reference src/lib/Force/Fermion/
 * force_F_Domainwall_eo.cpp:150-327): mode "H" computes force_udiv1_H(force,
 * zeta, eta), mode "Hdag" force_udiv1_Hdag(force, zeta, eta) with the
 * reference's argument order (eta first for Hdag: pass eta as `zeta_or_eta`).
 * force_lex: Field_G(Nvol, 4) layout, 18 reals per (site, mu).  alpha must be 1. */
int oracle_dwf_force_udiv1(oracle_dwf *op, const char *mode, double *force_lex,
                           const double *a, const double *b);
/* force_udiv(force, eta) = force_udiv1_H(H eta, eta) + force_udiv1_Hdag(eta, H eta). */
int oracle_dwf_force_udiv(oracle_dwf *op, double *force_lex, const double *eta);

/* Number of reals in one 5D half-lattice spinor. */
long oracle_dwf_field_size(const oracle_dwf *op);

#ifdef __cplusplus
}
#endif

#endif
