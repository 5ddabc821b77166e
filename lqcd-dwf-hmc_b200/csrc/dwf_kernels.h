// Host-side launch interface of the B200 domain-wall kernels.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include "dwf_common.cuh"
#include "dwf_chain.cuh"

namespace b200 {

struct HopParams;

// Geometry of one even/odd half lattice with Ls fifth-dimension slices.
struct Geom {
  int nx2, ny, nz, nt, ls;
  int vh;
};

// Site-local fifth-dimension maps (chiral-basis chains of dwf_chain.cuh).
enum SopKind {
  SOP_ID = 0, SOP_M5PRE, SOP_M5DAG, SOP_DEE, SOP_DEE_T, SOP_LU, SOP_LUDAG, SOP_G5R, SOP_R
};

// Parameters of the site-local fifth-dimension kernel:
//   o1 = ce * A(in) + cx1*X1 + cx2*X2,   o2 = B(o1)   (A = opa, B = opb)
// Scalars with a _dev pointer are multiplied by that device value at run time.
struct SopParams {
  const void* in;
  const void* x1;
  const void* x2;
  void* out1;
  void* out2;
  int opa, opb;
  double cx1, cx2, ce;
  const double* cx1_dev;
  const double* cx2_dev;
  const double* ce_dev;
  double* red;        // per-block partials of |o1|^2
  Geom g;
};

// CG vector update fused with the M5 pre-factor of the next hop:
//   x += alpha*p;  p = r + beta*p;  y = M5pre(p)   (alpha, beta device scalars)
struct CgUpdParams {
  void* x;
  void* p;
  const void* r;
  void* y;               // M5pre(p) for the next hop; null when M5pre is the identity
  const double* alpha;
  const double* beta;
  Geom g;
};

// Fifth-dimension chain coefficients of one operator in both arithmetic types.
struct ChainCoefs {
  ChainCoef<double> d;
  ChainCoef<float> f;
  ChainCoef<double> dee_d;   // D_ee: b -> b(4-M0)+1, c -> c(4-M0)-1
  ChainCoef<float> dee_f;
};

// Multishift CG (reference src/lib/Solver/ashiftsolver_CG-tmpl.h:216-286).
// Device state: scalars MS_* and per-shift arrays of kMaxShift entries.
constexpr int kMaxShift = 32;
enum MsScalar {
  MS_RR = 0, MS_RR_NEW, MS_PQ, MS_BETA, MS_ALPHA, MS_ALPHA_P, MS_BETA_P, MS_PP0,
  MS_SNORM, MS_SIGMA0, MS_TOL2, MS_NACT,
  MS_DONE,      // 0 while iterating; 1 converged, 2 NaN, 3 iteration cap (set by MSS_PRUNE)
  MS_ITER,      // iterations completed (counted on the device)
  MS_MAXITER,
  MS_WIN,       // windowed mode: residuals stored in the current window
  MS_NACTW,     // windowed mode: active shifts when the window opened
  MS_WSIZE,     // window length m (0: every shift updated every iteration)
  MS_N = 18
};
// per-shift arrays follow the scalars: [MS_N + a*kMaxShift + i]
enum MsArray { MSA_ZETA1 = 0, MSA_ZETA2, MSA_CSH2, MSA_BETAS, MSA_ALPHAS, MSA_ZETA, MSA_PP, MSA_COUNT };
// Windowed mode ("deferred shift updates"): the residuals r_0..r_(m-1) of m
// iterations are kept, and each shift carries coefficient vectors so that
//   p_i = PC[0] p_i(window start) + sum_l PC[1+l] r_l
//   x_i = x_i(window start) + XC[0] p_i(window start) + sum_l XC[1+l] r_l;
// the fields are touched once per window instead of once per iteration.
constexpr int kMaxWin = 16;
constexpr int kMsCoef = MS_N + MSA_COUNT * kMaxShift;                 // PC[i][0..m]
constexpr int kMsXCoef = kMsCoef + kMaxShift * (kMaxWin + 1);         // XC[i][0..m]
constexpr int kMsStateSize = kMsXCoef + kMaxShift * (kMaxWin + 1);

struct MsUpdParams {
  void* const* xs;       // device array [nshift] of solution fields
  void* const* ps;       // device array [nshift] of search directions
  const void* r;
  void* y0;              // M5pre(p_0) for the next hop (null: M5pre is the identity)
  const double* st;      // multishift state (MS_*, MSA_*)
  double* red;           // partials [kMaxShift][nblocks] of |p_i|^2
  int nblocks;
  Geom g;
  void* const* win;      // windowed mode: device array [kMaxWin] of residual slots (else null)
  void* p0s;             // windowed mode with x_0 deferred to the flush: p_0 at the window's
                         // start (else null; x_0 is then updated every iteration)
};
cudaError_t launch_ms_update(int prec, const MsUpdParams& p, const ChainCoefs& c, cudaStream_t st);
// Windowed mode: once the window is full (or the solve is over) apply the
// stored residuals to every shift that was active in the window (FP64), then
// reset the window (single-block kernel).
cudaError_t launch_ms_flush(const MsUpdParams& p, cudaStream_t st);
cudaError_t launch_ms_window_reset(double* st, cudaStream_t stream);
enum MsStep { MSS_BETA = 0, MSS_ALPHA = 1, MSS_PRUNE = 2 };
// scalar steps: MSS_BETA sums the K2 partials (pq) -> beta; MSS_ALPHA sums
// the K4 partials (rr_new) -> alpha and the per-shift zeta recurrence;
// MSS_PRUNE sums per-shift |p_i|^2 and drops converged shifts.
cudaError_t launch_ms_scalar(int step, const double* partials, int n, double* st, int nshift,
                             cudaStream_t stream);

// Fermion force terms (force.cu): for the sites x of parity ieo and mu = 0..3,
//   F_mu(x) = beta F_mu(x) + coef sum_s sum_spin
//             ( [(1 - g_mu) Y1(x+mu)]_c1 conj(Z1(x))_c2 + [(1 + g_mu) Y2(x+mu)]_c1 conj(Z2(x))_c2 )
// (either term may be absent), into the lexical Field_G(Nvol, 4) force.
struct ForceParams {
  const void* y1;
  const void* z1;
  const void* y2;
  const void* z2;
  double* force;
  double coef, beta;
  int ieo, vh, nx2, ny, nz, nt, ls;
  double bc[4];
};
cudaError_t launch_force(const ForceParams& p, cudaStream_t st);

// number of blocks the reductions of each launcher produce
int hop_grid(int ls, int vh);
int site_s_grid(int ls, int vh);
constexpr int kSiteSBlock = 128;


// Hop kernel dispatch (prec = storage precision of in/out fields; the hop
// direction (plain or gamma5-sandwiched dagger) follows from p.epi).
cudaError_t launch_hop(int prec, const HopParams& p, const ChainCoefs& c, cudaStream_t st);
cudaError_t launch_cg_update(int prec, const CgUpdParams& p, const ChainCoefs& c, cudaStream_t st);
cudaError_t launch_sop(int prec, const SopParams& p, const ChainCoefs& c, cudaStream_t st);


// y = a*x + b*y over the whole field (a, b optionally scaled by device values)
cudaError_t launch_axpby(int prec, const Geom& g, void* y, const void* x, double a,
                         const double* a_dev, double b, const double* b_dev, cudaStream_t st);
// partial sums of <x,y> (real part, double accumulation) into red[grid]
cudaError_t launch_dot(int prec, const Geom& g, const void* x, const void* y, double* red,
                       cudaStream_t st);
cudaError_t launch_convert(int pout, void* out, int pin, const void* in, const Geom& g,
                           cudaStream_t st);
cudaError_t launch_from_corelib(int prec, void* out, const double* in_dev, const Geom& g,
                                cudaStream_t st);
// parity ieo of a full-lattice lexical Field(24, Nvol, Ls) on the device
cudaError_t launch_from_lex_parity(int prec, void* out, const double* lex_dev, int ieo, const Geom& g,
                                  cudaStream_t st);
cudaError_t launch_to_corelib(int prec, double* out_dev, const void* in, const Geom& g,
                              cudaStream_t st);
// lexical links (corelib Field_G layout) -> even/odd links in link format lf
// (LINK_F64_18 with the boundary phases bc multiplied into the edge links)
cudaError_t launch_links_from_lex(int lf, void* out, const double* u_lex_dev, const Geom& g,
                                  const int bc[4], cudaStream_t st);

// out[0] = sum(partials[0..n)); op selects a solver scalar update afterwards:
enum FinalizeOp {
  FIN_SUM = 0,          // out[0] = s
  FIN_CG_ALPHA = 1,     // sc[PQ] = s; sc[ALPHA] = sc[RR] / s
  FIN_CG_BETA = 2,      // sc[BETA] = s / sc[RR]; sc[RR] = s
};
enum CgScalar { SC_RR = 0, SC_PQ = 1, SC_ALPHA = 2, SC_BETA = 3, SC_RR_NEW = 4, SC_N = 8 };
cudaError_t launch_finalize(const double* partials, int n, double* out, int op, cudaStream_t st);

size_t link_bytes(int lf, size_t vh);

// Complex FP64 BLAS on n complex numbers (double2), used by the flexible CG.
// launch_zdot: out = <x, y> = sum conj(x) y, or sign * <x, y> / Re(den[0])
// when den is given (partial: zblas_blocks() double2 scratch).
int zblas_blocks();
cudaError_t launch_zdot(const void* x, const void* y, size_t n, void* partial, void* out,
                        const void* den, double sign, cudaStream_t st);
cudaError_t launch_zaxpy(void* y, const void* x, size_t n, const void* c, cudaStream_t st);
// Up to kZMaxMulti fields at once (passed by value).
constexpr int kZMaxMulti = 8;
struct ZMulti {
  const double2* v[kZMaxMulti];
  int m;
};
// out[j] = sign * <Q_j, z> / Re(den[j]) for j < q.m in one pass over z
// (partial: zblas_blocks() * kZMaxMulti double2 scratch).
cudaError_t launch_zmdot(const ZMulti& q, const void* z, size_t n, void* partial, void* out,
                         const void* den, double sign, cudaStream_t st);
// y = z + sum_j c[j] P_j in one pass
cudaError_t launch_zmaxpy(void* y, const void* z, const ZMulti& pv, const void* c, size_t n,
                          cudaStream_t st);
// x += alpha p ; r -= alpha q ; partial[block] = |r|^2 (zblas_blocks() doubles)
cudaError_t launch_zcg_update(void* x, void* r, const void* p, const void* q, size_t n,
                              const void* alpha, double* partial, cudaStream_t st);

}  // namespace b200
