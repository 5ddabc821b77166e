/*
 * b200dwf -- C ABI of the B200-native even/odd 5D domain-wall fermion hot
 * path (operator, solvers) that stands in for the reference's flat device
 * kernel layer `namespace BridgeACC` and the classes built on it.
 *
 * Conventions shared by every entry point
 *   - Return value: 0 on success, a negative B200_E* code on failure; the
 *     message of the last failure on the calling thread is b200_last_error().
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).
 *   - Fields are device buffers of b200_dwf_field_bytes(op, prec) bytes holding
 *     one even/odd 5D half-lattice spinor (Nvol/2 sites x Ls) in the library's
 *     HBM layout; convert()/reverse() move data to and from the reference's
 *     host layout Field(24, Nvol/2, Ls):
 *         ri + 2*(color + 3*spin) + 24*(site_eo + Nvol2*s).
 *   - prec: B200_F64, B200_F32, B200_F16 (per-(site,s) scaled fp16 storage,
 *     fp32 arithmetic) or B200_BF16 (same with bf16 storage).
 *
 * Reference interfaces each group replaces (paths relative to the reference
 * tree; the reference's own header is src/lib_alt_Accel/BridgeOpenACC/
 * bridgeACC_Domainwall.h:14-495 for the kernels):
 */
#ifndef B200DWF_H
#define B200DWF_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  B200_F64 = 0,
  B200_F32 = 1,
  B200_F16 = 2,
  B200_BF16 = 3
};

enum {
  B200_OK = 0,
  B200_EINVAL = -1,     /* invalid argument / unsupported size */
  B200_ECUDA = -2,      /* CUDA runtime error */
  B200_ENOMEM = -3,     /* device allocation failed */
  B200_ENOCONV = -4     /* solver did not converge within its iteration cap */
};

typedef struct b200_dwf b200_dwf_t;

/* Message of the last error on this thread (never NULL). */
const char *b200_last_error(void);

/* Select the CUDA device of this process: device = rank % ndev + offset.
 * Replaces DeviceManager_OpenACC::init
 * (src/lib_alt_Accel/ResourceManager/deviceManager_OpenACC.cpp:31-50). */
int b200_init(int rank, int device_offset);

/* ---------------------------------------------------------------- operator
 * AFopr_Domainwall_5din_eo construction and parameters
 * (src/lib_alt_Accel/Fopr/afopr_Domainwall_5din_eo-tmpl.h:31-147 init,
 *  :330-405 set_parameters, :410-477 set_precond_parameters).
 * lattice = {Nx, Ny, Nz, Nt} (Nx even), Ls in {4, 6, 8, 12, 16},
 * b, c: Ls Moebius coefficients (NULL = Shamir b=1, c=0), alpha: Neff alpha,
 * bc: boundary phases {bx, by, bz, bt} (1 periodic, -1 antiperiodic, 0 open). */
int b200_dwf_create(b200_dwf_t **op, const int lattice[4], int Ls, double mq,
                    double M0, const double *b, const double *c, double alpha,
                    const int bc[4]);
int b200_dwf_destroy(b200_dwf_t *op);

/* set_config(Field *U) + convert_gauge: lexical links in the reference
 * Field_G(Nvol, 4) host layout ri + 2*(col + 3*row) + 18*(site + Nvol*mu)
 * (afopr_Domainwall_5din_eo-tmpl.h:514-551).  Builds the links for every
 * precision the operator is applied in. */
int b200_dwf_set_config(b200_dwf_t *op, const double *u_lex_host, void *stream);
/* Same, from a device buffer of the same layout. */
int b200_dwf_set_config_device(b200_dwf_t *op, const double *u_lex_dev, void *stream);

/* Bytes of one field of this operator in precision prec. */
size_t b200_dwf_field_bytes(const b200_dwf_t *op, int prec);
/* Number of reals in the reference host layout (24 * Nvol/2 * Ls). */
size_t b200_dwf_field_nreal(const b200_dwf_t *op);

/* convert(AFIELD&, const Field&) / reverse(Field&, const AFIELD&)
 * (afopr_Domainwall_5din_eo-tmpl.h:555-620): host double array in the
 * reference layout <-> device field.  Synchronous on `stream`. */
int b200_field_convert(b200_dwf_t *op, int prec, void *v_dev, const double *w_host,
                       void *stream);
int b200_field_reverse(b200_dwf_t *op, int prec, double *v_host, const void *w_dev,
                       void *stream);   /* also reports the plan's error word */
/* Asynchronous convert / reverse for pipelined host transfers (no reference
 * counterpart: the reference's convert/reverse are synchronous).  The host
 * field must be page-locked and stay untouched until `stream` has passed the
 * call.  Each direction has a ring of two device staging fields; a slot is
 * reused only after its previous transfer finished (a device-side wait), so
 * an upload on one stream and a download on another overlap on the two
 * copy directions. */
int b200_field_convert_async(b200_dwf_t *op, int prec, void *v_dev, const double *w_host,
                             void *stream);
int b200_field_reverse_async(b200_dwf_t *op, int prec, double *v_host, const void *w_dev,
                             void *stream);
/* The sites of parity ieo of a full-lattice lexical Field(24, Nvol, Ls) on
 * the device into a field (Index_eo::convertField(v, w_lex, ieo),
 * src/lib/Field/index_eo.cpp), asynchronous on `stream`: the heatbath's
 * lexical noise (action_F_Ratio_eo.cpp:70-78) without a separate gather. */
int b200_field_convert_lex_device(b200_dwf_t *op, int prec, void *v_dev, const double *w_lex_dev,
                                  int ieo, void *stream);
/* convert() from a field already on the device (w_dev: reference layout,
 * 24 * Nvol/2 * Ls doubles), asynchronous on `stream`: the heatbath noise
 * drawn by b200_rng_gauss_lex goes to the operator without a host copy. */
int b200_field_convert_device(b200_dwf_t *op, int prec, void *v_dev, const double *w_dev,
                              void *stream);

/* mult / mult_dag (afopr_Domainwall_5din_eo-tmpl.h:634-767).  mode is one of
 *   "D" "Ddag" "DdagD" "H" "Hdag" "Deo" "Doe" "Dee" "Doo" "Dee_inv" "Doo_inv"
 *   "gm5R" "R"
 * dag != 0 selects mult_dag.  v and w are distinct fields of precision prec.
 * Synchronous by default, like the reference's mult (its OpenACC launches
 * return after the kernels, mult_Domainwall_5din_eo_openacc-inc.h): the call
 * waits for its kernels and reports a bulk-copy wait that gave up as
 * B200_ECUDA (the output is then not written); see b200_dwf_set_async. */
int b200_dwf_mult(b200_dwf_t *op, int prec, void *v, const void *w,
                  const char *mode, int dag, void *stream);

/* Asynchronous calls (async != 0): b200_dwf_mult and the b200_dwf_force_*
 * entry points return once their kernels are queued on `stream`.  A hop that
 * gave up waiting for its bulk copies then surfaces at the next synchronising
 * call on this plan (b200_field_reverse, norm2/dot, the solvers) or at
 * b200_dwf_check_error.  No reference counterpart: the reference's launches
 * are synchronous.  Default 0. */
int b200_dwf_set_async(b200_dwf_t *op, int async_calls);
/* Waits for `stream`, then reports (B200_ECUDA) and clears the plan's device
 * error word of the hop kernels' bounded waits; 0 when it is clear. */
int b200_dwf_check_error(b200_dwf_t *op, void *stream);
/* Test hook of the failure path (host-set; no reference counterpart): every
 * bulk-copy (TMA-fed) hop launched by this plan treats its wait for hop
 * direction `direction` (0..7 = x+, x-, y+, y-, z+, z-, t+, t-) as if its
 * bound had run out: it sets the error word, still waits (with the long
 * drain bound) for the copies it has in flight, and returns without writing
 * its outputs.  Hops fed by plain loads have no waits and are unaffected.
 * -1 switches it off (the default). */
int b200_dwf_inject_wait_failure(b200_dwf_t *op, int direction);

/* Halo exchange for a lattice split along t over several ranks (replaces the
 * reference's per-hop face exchange, afopr_Domainwall_5din_eo-tmpl.h:998-1101
 * and 1126-1228 over the MPI channels of src/lib/Communicator/MPI/
 * channel.cpp:36-150).  A rank owning nt_loc slices (even) creates its plan
 * on the lattice {Lx, Ly, Lz, nt_loc + 2}, periodic in t, whose slices are its
 * own nt_loc slices, then the next rank's first slice, then the previous
 * rank's last slice; the global t boundary phase is folded into the global
 * last slice's t links by the caller.  The stencils then read the previous
 * rank's slice through the t wrap, and every site keeps its global parity.
 * Before each hop, and before the force kernels, the plan calls
 * fn(ctx, field, prec, stream) for every field they read at neighbouring
 * sites; fn must fill that field's two ghost slices (the t slowest index, so
 * each slice is one contiguous range of (Lx Ly Lz / 2) site columns) from the
 * neighbours' interior edge slices, ordered after the work already queued on
 * `stream`, and return 0.  The hops leave the output's ghost slices
 * unwritten (or, where they also reduce |out|^2, not meaningful).
 * With a hook set, the solvers and the learned preconditioner refuse the
 * plan (B200_EINVAL), and b200_field_norm2/dot cover the whole extended
 * lattice.  fn = NULL removes the hook. */
typedef int (*b200_halo_fn)(void *ctx, void *field, int prec, void *stream);
int b200_dwf_set_halo_exchange(b200_dwf_t *op, b200_halo_fn fn, void *ctx);
/* The same exchange in two halves, overlapped with the interior as the
 * reference overlaps its bulk hop with the face transfer
 * (afopr_Domainwall_5din_eo-tmpl.h:998-1101): start(ctx, field, prec, stream)
 * begins filling the ghost slices, ordered after the work on `stream`, and
 * returns; finish(...) makes `stream` wait until they are filled.  A hop
 * then launches the sites whose t neighbours are the rank's own (t = 1 ..
 * nt-2) between the two calls and the two edge slices after finish; the
 * force kernels call both before they run.  Needs nt >= 2 own slices.
 * Replaces a hook set by b200_dwf_set_halo_exchange; (NULL, NULL) removes
 * both. */
int b200_dwf_set_halo_exchange_split(b200_dwf_t *op, b200_halo_fn start, b200_halo_fn finish,
                                     void *ctx);

/* ---------------------------------------------------------------- fields
 * AField<REAL, ACCEL> BLAS (src/lib_alt_Accel/Field/afield-tmpl.h:637-720 ->
 * BridgeOpenACC/src/afield_openacc-inc.h:130-355).  norm2/dot accumulate in
 * double and return synchronously. */
int b200_field_axpby(b200_dwf_t *op, int prec, void *y, double a, const void *x,
                     double b, void *stream);                  /* y = a x + b y */
int b200_field_norm2(b200_dwf_t *op, int prec, const void *x, double *result,
                     void *stream);
int b200_field_dot(b200_dwf_t *op, int prec, const void *x, const void *y,
                   double *result, void *stream);              /* Re <x, y> */
int b200_field_copy_convert(b200_dwf_t *op, int prec_out, void *out, int prec_in,
                            const void *in, void *stream);     /* convert_h */

/* ---------------------------------------------------------------- solvers
 * ASolver_CG on DdagD, zero initial guess (src/lib_alt/Solver/
 * asolver_CG-tmpl.h:118-234): stops when |r|^2/|b|^2 < tol2; returns the
 * iteration count and diff = sqrt(|DdagD x - b|^2 / |b|^2) from a true
 * residual.  Returns B200_ENOCONV (x still written) if maxiter is reached. */
int b200_cg_solve(b200_dwf_t *op, int prec, void *x, const void *b, int maxiter,
                  double tol2, int *nconv, double *diff, void *stream);

/* AShiftsolver_CG on DdagD + sigma_i, FP64 (src/lib/Solver/
 * ashiftsolver_CG-tmpl.h:89-329, used by AFopr_Rational::mult src/lib/Fopr/
 * afopr_Rational-tmpl.h:181-219 and AForce_F_Rational_Ratio::force_udiv_impl
 * src/lib_alt/Force/Fermion/aforce_F_Rational_Ratio-tmpl.h:345-460).
 * x: nshift (<= 32) device fields; converged shifts are dropped as in the
 * reference.  nconv = iterations (the reference logs iterations - 1);
 * diff = max_i sqrt(|(DdagD + sigma_i) x_i - b|^2 / |b|^2). */
int b200_shiftcg_solve(b200_dwf_t *op, void *const *x, const double *sigma, int nshift,
                       const void *b, int maxiter, double tol2, int *nconv, double *diff,
                       void *stream);
/* Work fields, the shifted directions and the residual window are per-call
 * workspace shared by all plans of one device and geometry (vh, Ls): plans of
 * one geometry must not run calls concurrently on different streams.
 * Window m of the multishift solver's deferred shift updates (default 16):
 * the residuals of m iterations stay in HBM (m extra fields) and every shift's
 * x_i, p_i are updated once per window; 0 updates every shift every
 * iteration, as AShiftsolver_CG::solve_step does
 * (src/lib/Solver/ashiftsolver_CG-tmpl.h:216-286).  m <= 16. */
int b200_shiftcg_set_window(b200_dwf_t *op, int window);

/* Fprop_alt_Standard_eo_Richardson::invert_DdagD_even
 * (src/lib_alt/Measurements/Fermion/fprop_alt_Standard_eo_Richardson-tmpl.h:
 * 27-102, 460-481): ASolver_Richardson<double> (asolver_Richardson-tmpl.h:
 * 131-213) preconditioned by APrecond_Mixedprec (aprecond_Mixedprec-tmpl.h:
 * 55-108) around a zero-start inner CG on DdagD in inner_prec (B200_F32, or
 * B200_F16/B200_BF16 scaled storage with fp32 arithmetic); x, b are FP64
 * fields.  The reference's inner stop is tol2_inner = 1e-8.  Returns outer and
 * total inner iteration counts and diff = sqrt(|r|^2/|b|^2) of the FP64
 * residual. */
int b200_richardson_solve(b200_dwf_t *op, int inner_prec, void *x, const void *b,
                          int maxiter, double tol2, int maxiter_inner, double tol2_inner,
                          int *nconv, int *nconv_inner, double *diff, void *stream);
/* use_initial_guess of the reference's solvers (Solver_CG::set_parameters,
 * src/lib/Solver/solver_CG.cpp; ASolver_Richardson, src/lib_alt/Solver/
 * asolver_Richardson-tmpl.h:131-213): when set, b200_cg_solve and
 * b200_richardson_solve start from the x passed in instead of zero (CG runs on
 * the residual equation and adds the correction).  The stopping rule stays
 * |b - DdagD x|^2 / |b|^2 < tol2.  Default 0, as in the reference's inputs. */
int b200_solver_set_initial_guess(b200_dwf_t *op, int use);

/* Allocation-free |x|^2 for callers that cannot allocate device memory: code
 * running under a host framework that owns all device memory through its own
 * pool (an allocation behind its back can fail or exhaust what the pool
 * planned for), or a caller on a GPU whose memory is already committed to
 * resident fields.  It needs no operator plan (a plan owns its reduction
 * scratch): pass the field x (precision prec, nsite 4D half-lattice sites,
 * Ls = ls) and a host pointer for the result.  No counterpart in the
 * reference (its norm2 always runs on fields that an operator allocated).
 *   - Scratch is a fixed 512 KiB device array inside the library, held by
 *     every GPU that loads it until the process exits; fields larger than
 *     8,388,608 (site, s) pairs are rejected with B200_EINVAL.
 *   - The first call on each device looks the array up (once per device).
 *   - All calls on a device share the array: calls that overlap on the GPU
 *     (different streams, no ordering between them) race and give wrong sums.
 *   - Calls no cudaMalloc/cudaFree; synchronous on `stream`. */
int b200_field_norm2_noalloc(int prec, const void *x, long nsite, int ls,
                             double *result, void *stream);

/* ---------------------------------------------------------------- flat vectors
 * Plan-free vector operations on device arrays of n reals (prec 0: double,
 * 1: float), for field containers that hold a library field as a flat
 * array: the reference-side AField<REAL, B200> shell.  They replace the
 * BridgeACC vector functions (src/lib_alt_Accel/BridgeOpenACC/src/
 * afield_openacc-inc.h:14-446).  Element-wise work does not depend on the
 * layout; complex forms act on adjacent (re, im) pairs (n even).
 * Reductions accumulate in double and return synchronously on `stream`;
 * reductions from several host threads on one device take turns (they share
 * the device's scratch). */
int b200_blas_axpby(int prec, size_t n, double a, const void *x, double b, void *y,
                    void *stream);                         /* y = a x + b y (b = 0: y not read) */
int b200_blas_caxpby(int prec, size_t n, double ar, double ai, const void *x, double br,
                     double bi, void *y, void *stream);    /* complex pairs */
int b200_blas_fill(int prec, size_t n, double value, void *y, void *stream);
int b200_blas_dot(int prec, size_t n, const void *x, const void *y, double *result,
                  void *stream);                           /* sum x_i y_i */
int b200_blas_dotc(int prec, size_t n, const void *x, const void *y, double *re, double *im,
                   void *stream);                          /* sum conj(x) y over pairs */
/* Precision copy of a field of nsite (site, Ls) columns between storage
 * precisions 0..3 (convert_h, afield_copy_openacc-inc.h:11-54): the storage
 * layouts differ per precision, so this is layout-aware. */
int b200_field_convert_prec(int prec_out, void *out, int prec_in, const void *in, long nsite,
                            int ls, void *stream);

/* ---------------------------------------------------------------- force
 * Force_F_Domainwall_eo::force_udiv1 (src/lib/Force/Fermion/
 * force_F_Domainwall_eo.cpp:170-318; Accel form AForce_F_Domainwall_5din_eo::
 * force_udiv1_H/Hdag, src/lib_alt_Accel/Force/Fermion/
 * aforce_F_Domainwall_5din_eo-tmpl.h:342-453) with the reference's argument
 * order: mode "H": a = zeta (= H eta), b = eta; mode "Hdag": a = eta,
 * b = zeta.  force: device array in the lexical Field_G(Nvol, 4) layout
 * (18 reals per (site, mu)), fully overwritten.  FP64 fields; the operator's
 * parameter_alpha must be 1 (as in the reference). */
int b200_dwf_force_udiv1(b200_dwf_t *op, const char *mode, double *force, const void *a,
                         const void *b, void *stream);
/* force_udiv(force, eta) = force_udiv1_H(H eta, eta) + force_udiv1_Hdag(eta, H eta)
 * (force_F_Domainwall_eo.cpp:150-167), fused: three hops and two force passes. */
int b200_dwf_force_udiv(b200_dwf_t *op, double *force, const void *eta, void *stream);
/* Accumulating form: force += scale * force_udiv1(mode "H"/"Hdag", a, b) or
 * force += scale * force_udiv(a) (mode "DdagD", b unused).  Replaces the
 * force_udiv + axpy pairs of the reference's ratio and rational forces
 * (Force_F_Rational_Ratio::force_udiv_impl, src/lib/Force/Fermion/
 * force_F_Rational_Ratio.cpp:253-292; Action_F_Ratio_eo::force,
 * src/lib/Action/Fermion/action_F_Ratio_eo.cpp:171-205). */
int b200_dwf_force_acc(b200_dwf_t *op, const char *mode, double *force, const void *a,
                       const void *b, double scale, void *stream);
/* The force entry points are synchronous like b200_dwf_mult (and report the
 * error word) unless the plan is switched to asynchronous calls. */

/* ---------------------------------------------------------------- stout
 * Stout smearing levels and the smeared-force Jacobian, on the device.
 * Director_Smear + Smear_APE + Projection_Stout_SU3 (src/lib/Smear/
 * director_Smear.cpp, smear_APE.cpp:108-140, projection_Stout_SU3.cpp:60-500;
 * alt driver Director_alt_Smear src/lib_alt/Smear/director_alt_Smear-tmpl.h:
 * 21-286) and ForceSmear_APE::force_udiv (src/lib/Smear/forceSmear_APE.cpp)
 * chained by AForce_F_Smeared_alt::mult_jacobian (src/lib_alt/Force/Fermion/
 * aforce_F_Smeared_alt-tmpl.h:170-191).  Links and forces: device arrays in
 * the lexical Field_G(Nvol, 4) layout. */
typedef struct b200_smear b200_smear_t;
int b200_smear_create(b200_smear_t **sm, const int lattice[4], double rho, int nsmear);
int b200_smear_destroy(b200_smear_t *sm);
/* set_config + smear: u = thin links (host if on_device == 0, else device). */
int b200_smear_set_config(b200_smear_t *sm, const double *u, int on_device, void *stream);
/* Device pointer of smearing level `level` (0 = thin links, nsmear = fully
 * smeared); NULL if out of range or no config was set. */
const double *b200_smear_config(b200_smear_t *sm, int level);
/* Copy of level `level` to host memory (18*4*Nvol doubles). */
int b200_smear_get_config(b200_smear_t *sm, int level, double *host_out, void *stream);
/* mult_jacobian: sigma (force w.r.t. the fully smeared links) is replaced in
 * place by the force w.r.t. the thin links. */
int b200_smear_jacobian(b200_smear_t *sm, double *sigma, void *stream);
/* AForce_F::mult_generator (src/lib_alt_Accel/Force/Fermion/aforce_F.cpp:62-75):
 * force <- -2 * (traceless anti-Hermitian part of U force), per link. */
int b200_force_mult_generator(const int lattice[4], double *force, const double *u, void *stream);

/* ---------------------------------------------------------------- gauge side of the HMC step
 * Device arrays in the lexical Field_G(Nvol, 4) layout (18 reals per link),
 * FP64.  Iwasaki / rectangle gauge action with beta, c_plaq, c_rect.
 * Force_G_Rectangle::force_core (src/lib/Force/Gauge/force_G_Rectangle.cpp:
 * 84-220): force = -(beta/3) TA(U_mu sum of staples^+), overwritten. */
int b200_gauge_force_rect(const int lattice[4], double beta, double c_plaq, double c_rect,
                          double *force, const double *u, void *stream);
/* Action_G_Rectangle::calcH (src/lib/Action/Gauge/action_G_Rectangle.cpp:97-200);
 * synchronous. */
int b200_gauge_action_rect(const int lattice[4], double beta, double c_plaq, double c_rect,
                           const double *u, double *H, void *stream);
/* Integrator_UpdateU::evolve (src/lib/HMC/integrator_UpdateU.cpp:79-86 ->
 * mult_exp_Field_G, SU_N::mat_exp, reunit_SU3): u <- exp(alpha iP) u in place,
 * Taylor order nprec, reunitarised. */
int b200_link_update(const int lattice[4], double alpha, const double *ip, double *u, int nprec,
                     void *stream);
/* Integrator_UpdateP::evolve (src/lib/HMC/integrator_UpdateP.cpp:44-66):
 * ip += eps * force. */
int b200_momentum_update(const int lattice[4], double eps, const double *force, double *ip,
                         void *stream);
/* HMC_General::calcH_P (src/lib/HMC/hmc_General.cpp:340-346): H = |iP|^2 / 2;
 * synchronous. */
/* iP = i sum_a h_a lambda_a on every link from Field(8, Nvol, 4) Gaussians h
 * (Langevin_Momentum::set_iP_SU3, src/lib/HMC/langevin_Momentum.cpp:150-210);
 * device arrays, asynchronous on `stream`. */
int b200_momentum_from_gauss(const int lattice[4], const double *h, double *ip, void *stream);
/* y = a x + b y over link/force fields (Field_G(Nvol, 4), 72 Nvol doubles);
 * b = 0 overwrites y without reading it.  The force sums of
 * Integrator_UpdateP (src/lib/HMC/integrator_UpdateP.cpp:44-66). */
int b200_links_axpby(const int lattice[4], double a, const double *x, double b, double *y,
                     void *stream);
int b200_momentum_energy(const int lattice[4], const double *ip, double *H, void *stream);

/* ---------------------------------------------------------------- learned preconditioner
 * No reference counterpart.  A 3-layer linear gauge-covariant 5D convolution
 * network N ~ (DdagD)^-1 for the even-parity system: channels 4 -> hidden ->
 * 4 per color (input channels = the 4 spins), 11 paths per layer (identity,
 * s+1, s-1 with open ends, the 8 link-transported 4D hops with the operator's
 * boundary phases), complex weights rounded to BF16, FP32 accumulation.  It
 * takes the place of an APrecond<AFIELD> (src/lib_alt/Solver/aprecond.h:
 * 28-47) in a flexible solver.  Fields r, z, e: device FP32 fields of the
 * operator (B200_F32 layout).  Weights: 2*b200_lp_nparams() floats, complex
 * interleaved, layer-major [layer][path][out][in]. */
typedef struct b200_lp b200_lp_t;
int b200_lp_create(b200_lp_t **lp, b200_dwf_t *op, int hidden, unsigned long long seed,
                   double init_noise);
int b200_lp_destroy(b200_lp_t *lp);
int b200_lp_nparams(const b200_lp_t *lp);
/* FP32 master weights (set resets the optimiser state); get with deployed != 0
 * returns the BF16-rounded weights the kernels use. */
int b200_lp_set_weights(b200_lp_t *lp, const float *w, int nfloat);
int b200_lp_get_weights(b200_lp_t *lp, float *w, int nfloat, int deployed);
/* z = N(r). */
int b200_lp_apply(b200_lp_t *lp, void *z, const void *r, void *stream);
/* For a pair with DdagD e = r: loss = |DdagD (N(r) - e)|^2 / |r|^2 (the
 * error of N measured in the residual norm) and its gradient
 * dL/dRe(w) + i dL/dIm(w), kept on the device (b200_lp_get_grad copies it
 * out).  Synchronous. */
int b200_lp_loss_grad(b200_lp_t *lp, const void *r, const void *e, double *loss, void *stream);
int b200_lp_get_grad(b200_lp_t *lp, float *g, int nfloat);
/* One Adam step (beta1 0.9, beta2 0.999, eps 1e-8) on the master weights. */
int b200_lp_adam_step(b200_lp_t *lp, double lr, void *stream);
/* `epochs` passes of loss_grad + adam_step over the pairs in a seeded
 * shuffled order; mean loss of the first and the last epoch.  A network that
 * has not taken a step yet first scales its last layer by the least-squares
 * factor Re<DdagD N r, r> / |DdagD N r|^2 of the first pair. */
int b200_lp_train(b200_lp_t *lp, int npairs, const void *const *r, const void *const *e,
                  int epochs, double lr, unsigned long long seed, double *loss_first,
                  double *loss_last, void *stream);
/* Plain CG (as b200_cg_solve, without the true residual) copying x after
 * iteration iters[j] into snaps[j] (fields of precision prec). */
int b200_cg_snapshots(b200_dwf_t *op, int prec, void *x, const void *b, int maxiter,
                      double tol2, int nsnap, const int *iters, void *const *snaps,
                      int *nconv, void *stream);
/* Flexible CG on DdagD preconditioned by lp: FP64 x, b; the new search
 * direction is A-orthogonalised against the last mtrunc (1..8) directions.
 * The FP64 true residual judges the result: if it misses tol2, plain CG on
 * the residual equation finishes from x (*nconv_fallback iterations, at most
 * 100000, independent of maxiter).  diff = sqrt(|DdagD x - b|^2 / |b|^2). */
int b200_fcg_solve(b200_dwf_t *op, b200_lp_t *lp, void *x, const void *b, int maxiter,
                   double tol2, int mtrunc, int *nconv, int *nconv_fallback, double *diff,
                   void *stream);

/* ---------------------------------------------------------------- heatbath noise
 * The benchmark driver's random numbers on the device (random_number_type
 * Mseries_parallel): RandomNumbers_parallel<RandomNumbers_Mseries>
 * (src/lib/Tools/randomNumbers_parallel-tmpl.h:160-300 init_2d,
 * set_lex_global_2d, gauss_lex_global, uniform_lex_global; streams
 * src/lib/Tools/randomNumbers_Mseries.cpp:32-150; Gaussian pairs
 * src/lib/Tools/randomNumbers.cpp:53-75).  One M-series stream per (z, t)
 * plane of the global lattice, each advancing across calls as in the
 * reference.  Fields are device buffers of nin * Nvol * nex doubles in the
 * corelib Field layout (component fastest, then lexical site, then extra
 * index).  The uniform numbers are the reference's bit for bit; the
 * Gaussians agree to the last bits of the device's log/sqrt/sin/cos.
 * create/reset compute the streams' start states on the host (the
 * reference's seeding and 1000 discarded numbers) and wait for the device. */
typedef struct b200_rng b200_rng_t;
int b200_rng_create(b200_rng_t **out, const int lattice[4], unsigned long seed);
int b200_rng_reset(b200_rng_t *rng, unsigned long seed);   /* RandomNumbers::reset */
/* gauss_lex_global(Field(nin, Nvol, nex)); nin even */
int b200_rng_gauss_lex(b200_rng_t *rng, double *v, int nin, int nex, void *stream);
/* uniform_lex_global: one number per site in component 0, the others 0 */
int b200_rng_uniform_lex(b200_rng_t *rng, double *v, int nin, int nex, void *stream);
int b200_rng_destroy(b200_rng_t *rng);

/* ---------------------------------------------------------------- tuning
 * Text table of the autotuner's choices (one line per geometry, precision and
 * kernel epilogue: chosen occupancy variant and its time per launch).  The
 * reference picks its kernel shape at compile time (NUM_WORKERS /
 * VECTOR_LENGTH, src/lib_alt_Accel/inline/define_params.h:35-36); here the
 * choice is measured on the first launch (disable with B200_AUTOTUNE=0). */
int b200_tuning_table(char *buf, size_t n);

#ifdef __cplusplus
}
#endif

#endif
