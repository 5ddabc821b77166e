/*
 * CPU oracle: even-odd 5D domain-wall operator, CG and multishift CG.
 *
 * TEST INFRASTRUCTURE ONLY -- a plain-C restatement of the reference Bridge++
 * corelib algorithm used to check the CUDA product path.  Every function cites
 * the reference file:line it follows (paths relative to the reference tree).
 *
 * Conventions (reference src/lib/Fopr/afopr_Domainwall_eo-tmpl.h):
 *   D_eo(w)  = (4-M0) * WilsonDeo_kappa( b*Wf(w) + c*V(w) ),  kappa=1/(8-2M0)
 *            = -1/2 * hop( b*Wf(w) + c*V(w) )                         (:764-826)
 *   hop(w)(x)= sum_mu bc*(1-g_mu) U_mu(x) w(x+mu) + bc*(1+g_mu) U_mu(x-mu)^+ w(x-mu)
 *              (src/lib/Fopr/Imp/fopr_Wilson_eo_impl.cpp:498-519, 714-1430)
 *   Wf(w)(s) = (alpha P+ + P-) w(0) at s=0, (P+ + alpha P-) w(Ls-1) at s=Ls-1,
 *              alpha w(s) in the bulk
 *   V(w)(s)  = Fup (1-g5) w(s+1) + Fdn (1+g5) w(s-1), Fup=Fdn=alpha/2 except
 *              Fup=-mq/2 at s=Ls-1 and Fdn=-mq/2 at s=0 (walls wrap in s).
 * Dirac gamma matrices: src/lib/Tools/gammaMatrixSet_Dirac.cpp:31-60.
 */
#include "dwf_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define NC 3
#define NSP 4
#define NIN 24  /* reals per 4D spinor site */
#define NDF 18  /* reals per link */

struct oracle_dwf {
  int L[4];
  int Nx2, Vh, V, Ls;
  double mq, M0, alpha;
  double *b, *c;
  int bc[4];
  double *dp, *dm, *e, *f;
  double g;
  double *ueo;            /* 18*(site + Vh*(ieo + 2*mu)) */
  double *w1, *w2, *w3, *w4;   /* scratch 5D fields */
};

/* ---- gamma matrices (Dirac representation), one non-zero per row ---- */
/* gcol[mu][i] column of the non-zero in row i, gre/gim its value.       */
static const int gcol[5][4] = {
  {3, 2, 1, 0},   /* gamma1 */
  {3, 2, 1, 0},   /* gamma2 */
  {2, 3, 0, 1},   /* gamma3 */
  {0, 1, 2, 3},   /* gamma4 */
  {2, 3, 0, 1},   /* gamma5 */
};
static const double gre[5][4] = {
  {0, 0, 0, 0},
  {-1, 1, 1, -1},
  {0, 0, 0, 0},
  {1, 1, -1, -1},
  {1, 1, 1, 1},
};
static const double gim[5][4] = {
  {-1, -1, 1, 1},
  {0, 0, 0, 0},
  {-1, 1, 1, -1},
  {0, 0, 0, 0},
  {0, 0, 0, 0},
};

/* out = gamma_mu * in  on one 4D spinor site (24 reals) */
static void gamma_mult(double *out, const double *in, int mu)
{
  for (int i = 0; i < NSP; ++i) {
    int j = gcol[mu][i];
    double vr = gre[mu][i], vi = gim[mu][i];
    for (int c = 0; c < NC; ++c) {
      double xr = in[2 * (c + 3 * j)], xi = in[2 * (c + 3 * j) + 1];
      out[2 * (c + 3 * i)]     = vr * xr - vi * xi;
      out[2 * (c + 3 * i) + 1] = vr * xi + vi * xr;
    }
  }
}

/* out += a*in + b5*gamma5*in on one site */
static void axpy_g5(double *out, double a, double b5, const double *in)
{
  double t[NIN];
  gamma_mult(t, in, 4);
  for (int k = 0; k < NIN; ++k) out[k] += a * in[k] + b5 * t[k];
}

/* u*v for a 3x3 complex matrix (row-major, 18 reals) on a color vector
 * stored with stride 2 (re,im) */
static void su3_mult(double *out, const double *u, const double *v)
{
  for (int i = 0; i < NC; ++i) {
    double re = 0, im = 0;
    for (int j = 0; j < NC; ++j) {
      double ur = u[2 * (j + 3 * i)], ui = u[2 * (j + 3 * i) + 1];
      re += ur * v[2 * j] - ui * v[2 * j + 1];
      im += ur * v[2 * j + 1] + ui * v[2 * j];
    }
    out[2 * i] = re;
    out[2 * i + 1] = im;
  }
}

static void su3_dag_mult(double *out, const double *u, const double *v)
{
  for (int i = 0; i < NC; ++i) {
    double re = 0, im = 0;
    for (int j = 0; j < NC; ++j) {
      double ur = u[2 * (i + 3 * j)], ui = -u[2 * (i + 3 * j) + 1];
      re += ur * v[2 * j] - ui * v[2 * j + 1];
      im += ur * v[2 * j + 1] + ui * v[2 * j];
    }
    out[2 * i] = re;
    out[2 * i + 1] = im;
  }
}

static double *fld(const oracle_dwf *op, double *base, int site, int s)
{
  return base + (size_t)NIN * (site + (size_t)op->Vh * s);
}

static const double *cfld(const oracle_dwf *op, const double *base, int site, int s)
{
  return base + (size_t)NIN * (site + (size_t)op->Vh * s);
}

long oracle_dwf_field_size(const oracle_dwf *op)
{
  return (long)NIN * op->Vh * op->Ls;
}

/* Coefficients of the LU decomposition of D_ee,
 * reference src/lib/Fopr/afopr_Domainwall_eo-tmpl.h:239-273. */
static void set_precond(oracle_dwf *op)
{
  int Ls = op->Ls;
  for (int s = 0; s < Ls; ++s) {
    op->dp[s] = op->alpha * (1.0 + op->b[s] * (4.0 - op->M0));
    op->dm[s] = op->alpha * (1.0 - op->c[s] * (4.0 - op->M0));
  }
  op->e[0] = op->mq * op->dm[Ls - 1] / op->dp[0];
  op->f[0] = op->mq * op->dm[0] / op->alpha;
  for (int s = 1; s < Ls - 1; ++s) {
    op->e[s] = op->e[s - 1] * op->dm[s - 1] / op->dp[s];
    op->f[s] = op->f[s - 1] * op->dm[s] / op->dp[s - 1];
  }
  op->g = op->e[Ls - 2] * op->dm[Ls - 2];
}

oracle_dwf *oracle_dwf_create(const int lattice[4], int Ls, double mq,
                              double M0, const double *b, const double *c,
                              double alpha, const int bc[4])
{
  if (Ls < 2 || lattice[0] % 2 != 0) return NULL;
  oracle_dwf *op = (oracle_dwf *)calloc(1, sizeof(oracle_dwf));
  memcpy(op->L, lattice, 4 * sizeof(int));
  op->V = lattice[0] * lattice[1] * lattice[2] * lattice[3];
  op->Vh = op->V / 2;
  op->Nx2 = lattice[0] / 2;
  op->Ls = Ls;
  op->mq = mq;
  op->M0 = M0;
  op->alpha = alpha;
  memcpy(op->bc, bc, 4 * sizeof(int));
  op->b = (double *)malloc(Ls * sizeof(double));
  op->c = (double *)malloc(Ls * sizeof(double));
  memcpy(op->b, b, Ls * sizeof(double));
  memcpy(op->c, c, Ls * sizeof(double));
  op->dp = (double *)malloc(Ls * sizeof(double));
  op->dm = (double *)malloc(Ls * sizeof(double));
  op->e = (double *)malloc(Ls * sizeof(double));
  op->f = (double *)malloc(Ls * sizeof(double));
  set_precond(op);
  op->ueo = (double *)calloc((size_t)NDF * op->V * 4, sizeof(double));
  size_t n = (size_t)NIN * op->Vh * Ls;
  op->w1 = (double *)calloc(n, sizeof(double));
  op->w2 = (double *)calloc(n, sizeof(double));
  op->w3 = (double *)calloc(n, sizeof(double));
  op->w4 = (double *)calloc(n, sizeof(double));
  return op;
}

void oracle_dwf_destroy(oracle_dwf *op)
{
  if (!op) return;
  free(op->b); free(op->c); free(op->dp); free(op->dm); free(op->e);
  free(op->f); free(op->ueo); free(op->w1); free(op->w2); free(op->w3);
  free(op->w4);
  free(op);
}

/* lexical -> even/odd links: U_eo[ieo][mu][site_eo] = U[mu][lex site],
 * site_eo = x/2 + Nx/2*(y + Ny*(z + Nz*t)), ieo = (x+y+z+t)%2
 * (reference src/lib/Field/index_eo.h:65-105, single rank). */
void oracle_dwf_set_links(oracle_dwf *op, const double *u_lex)
{
  const int *L = op->L;
  for (int mu = 0; mu < 4; ++mu)
    for (int t = 0; t < L[3]; ++t)
      for (int z = 0; z < L[2]; ++z)
        for (int y = 0; y < L[1]; ++y)
          for (int x = 0; x < L[0]; ++x) {
            int lex = x + L[0] * (y + L[1] * (z + L[2] * t));
            int ieo = (x + y + z + t) % 2;
            int seo = x / 2 + op->Nx2 * (y + L[1] * (z + L[2] * t));
            memcpy(op->ueo + (size_t)NDF * (seo + (size_t)op->Vh * (ieo + 2 * mu)),
                   u_lex + (size_t)NDF * (lex + (size_t)op->V * mu),
                   NDF * sizeof(double));
          }
}

/* Wilson hop, output parity ieo, no -kappa factor; when jgm5 the input and
 * output are sandwiched by gamma5 (the dagger hop).  Reference
 * src/lib/Fopr/Imp/fopr_Wilson_eo_impl.cpp:714-1430 (per-direction
 * projections), boundary phase bc at the lattice edge. */
static void hop(const oracle_dwf *op, double *out, const double *in, int ieo)
{
  const int *L = op->L;
  const int Ls = op->Ls;
#pragma omp parallel for schedule(static)
  for (int site = 0; site < op->Vh; ++site) {
    int ix2 = site % op->Nx2;
    int iyzt = site / op->Nx2;
    int y = iyzt % L[1];
    int z = (iyzt / L[1]) % L[2];
    int t = iyzt / (L[1] * L[2]);
    int keo = (ieo + y + z + t) % 2;
    int xc[4] = {2 * ix2 + keo, y, z, t};
    for (int s = 0; s < Ls; ++s) memset(fld(op, out, site, s), 0, NIN * sizeof(double));
    for (int mu = 0; mu < 4; ++mu) {
      for (int dir = 0; dir < 2; ++dir) {   /* 0: forward, 1: backward */
        int nc[4] = {xc[0], xc[1], xc[2], xc[3]};
        double ph = 1.0;
        if (dir == 0) {
          if (nc[mu] == L[mu] - 1) { nc[mu] = 0; ph = op->bc[mu]; } else nc[mu] += 1;
        } else {
          if (nc[mu] == 0) { nc[mu] = L[mu] - 1; ph = op->bc[mu]; } else nc[mu] -= 1;
        }
        int nb = nc[0] / 2 + op->Nx2 * (nc[1] + L[1] * (nc[2] + L[2] * nc[3]));
        const double *u = (dir == 0)
          ? op->ueo + (size_t)NDF * (site + (size_t)op->Vh * (ieo + 2 * mu))
          : op->ueo + (size_t)NDF * (nb + (size_t)op->Vh * ((1 - ieo) + 2 * mu));
        double sg = (dir == 0) ? -1.0 : 1.0;   /* (1 - g_mu) forward, (1 + g_mu) backward */
        for (int s = 0; s < Ls; ++s) {
          const double *w = cfld(op, in, nb, s);
          double tmp[NIN], gt[NIN];
          for (int sp = 0; sp < NSP; ++sp) {
            if (dir == 0) su3_mult(tmp + 6 * sp, u, w + 6 * sp);
            else su3_dag_mult(tmp + 6 * sp, u, w + 6 * sp);
          }
          gamma_mult(gt, tmp, mu);
          double *o = fld(op, out, site, s);
          for (int k = 0; k < NIN; ++k) o[k] += ph * (tmp[k] + sg * gt[k]);
        }
      }
    }
  }
}

static void g5_field(const oracle_dwf *op, double *out, const double *in)
{
  size_t n = (size_t)op->Vh * op->Ls;
  for (size_t i = 0; i < n; ++i) gamma_mult(out + NIN * i, in + NIN * i, 4);
}

/* wall factor Wf: (alpha P+ + P-) at s=0, (P+ + alpha P-) at s=Ls-1, alpha
 * in the bulk (afopr_Domainwall_eo-tmpl.h:790-808) */
static void wall(const oracle_dwf *op, double *out, const double *in, int s, double scale)
{
  double a = op->alpha;
  if (s == 0) {
    for (int k = 0; k < NIN; ++k) out[k] = 0;
    axpy_g5(out, scale * 0.5 * (1 + a), scale * 0.5 * (a - 1), in);
  } else if (s == op->Ls - 1) {
    for (int k = 0; k < NIN; ++k) out[k] = 0;
    axpy_g5(out, scale * 0.5 * (1 + a), scale * 0.5 * (1 - a), in);
  } else {
    for (int k = 0; k < NIN; ++k) out[k] = scale * a * in[k];
  }
}

/* out(s) = cw*Wf(in)(s) + cv*V(in)(s), cw/cv per s.  Shared by D_eo's M5
 * pre-factor (cw=b, cv=c) and D_ee (cw=b(4-M0)+1, cv=c(4-M0)-1). */
static void m5_apply(const oracle_dwf *op, double *out, const double *in,
                     const double *cw, const double *cv)
{
  const int Ls = op->Ls;
#pragma omp parallel for schedule(static)
  for (int site = 0; site < op->Vh; ++site) {
    for (int s = 0; s < Ls; ++s) {
      double *o = fld(op, out, site, s);
      wall(op, o, cfld(op, in, site, s), s, cw[s]);
      int sup = (s + 1) % Ls, sdn = (s - 1 + Ls) % Ls;
      double fup = (s == Ls - 1) ? -0.5 * op->mq : 0.5 * op->alpha;
      double fdn = (s == 0) ? -0.5 * op->mq : 0.5 * op->alpha;
      axpy_g5(o, cv[s] * fup, -cv[s] * fup, cfld(op, in, site, sup));
      axpy_g5(o, cv[s] * fdn, cv[s] * fdn, cfld(op, in, site, sdn));
    }
  }
}

/* adjoint of m5_apply: out = sum over s of the transposed couplings
 * (afopr_Domainwall_eo-tmpl.h:830-898 for D_eo^+, :958-1016 for D_ee^+) */
static void m5_apply_dag(const oracle_dwf *op, double *out, const double *in,
                         const double *cw, const double *cv)
{
  const int Ls = op->Ls;
#pragma omp parallel for schedule(static)
  for (int site = 0; site < op->Vh; ++site) {
    for (int s = 0; s < Ls; ++s) memset(fld(op, out, site, s), 0, NIN * sizeof(double));
    for (int s = 0; s < Ls; ++s) {
      const double *z = cfld(op, in, site, s);
      double t[NIN];
      wall(op, t, z, s, cw[s]);
      double *o = fld(op, out, site, s);
      for (int k = 0; k < NIN; ++k) o[k] += t[k];
      int sup = (s + 1) % Ls, sdn = (s - 1 + Ls) % Ls;
      double fup = (sup == 0) ? -0.5 * op->mq : 0.5 * op->alpha;
      double fdn = (sdn == Ls - 1) ? -0.5 * op->mq : 0.5 * op->alpha;
      axpy_g5(fld(op, out, site, sup), cv[s] * fup, -cv[s] * fup, z);
      axpy_g5(fld(op, out, site, sdn), cv[s] * fdn, cv[s] * fdn, z);
    }
  }
}

static void D_eo(oracle_dwf *op, double *out, const double *in, int ieo)
{
  m5_apply(op, op->w4, in, op->b, op->c);
  hop(op, out, op->w4, ieo);
  size_t n = (size_t)NIN * op->Vh * op->Ls;
  for (size_t i = 0; i < n; ++i) out[i] *= -0.5;
}

static void Ddag_eo(oracle_dwf *op, double *out, const double *in, int ieo)
{
  size_t n = (size_t)NIN * op->Vh * op->Ls;
  g5_field(op, out, in);
  hop(op, op->w4, out, ieo);
  g5_field(op, out, op->w4);
  for (size_t i = 0; i < n; ++i) out[i] *= -0.5;
  memcpy(op->w4, out, n * sizeof(double));
  m5_apply_dag(op, out, op->w4, op->b, op->c);
}

static void D_ee(oracle_dwf *op, double *out, const double *in, int dag)
{
  double *cw = (double *)malloc(op->Ls * sizeof(double));
  double *cv = (double *)malloc(op->Ls * sizeof(double));
  for (int s = 0; s < op->Ls; ++s) {
    cw[s] = op->b[s] * (4.0 - op->M0) + 1.0;
    cv[s] = op->c[s] * (4.0 - op->M0) - 1.0;
  }
  if (dag) m5_apply_dag(op, out, in, cw, cv); else m5_apply(op, out, in, cw, cv);
  free(cw);
  free(cv);
}

/* L^{-1}: afopr_Domainwall_eo-tmpl.h:1022-1062 */
static void L_inv(const oracle_dwf *op, double *v, const double *w)
{
  const int Ls = op->Ls;
#pragma omp parallel for schedule(static)
  for (int site = 0; site < op->Vh; ++site) {
    double y[NIN];
    memcpy(fld(op, v, site, 0), cfld(op, w, site, 0), NIN * sizeof(double));
    for (int k = 0; k < NIN; ++k) y[k] = op->e[0] * cfld(op, w, site, 0)[k];
    for (int s = 1; s < Ls; ++s) {
      double *vs = fld(op, v, site, s);
      memcpy(vs, cfld(op, w, site, s), NIN * sizeof(double));
      double a = 0.5 * op->dm[s] / op->dp[s - 1];
      axpy_g5(vs, a, a, fld(op, v, site, s - 1));
      if (s < Ls - 1) {
        for (int k = 0; k < NIN; ++k) y[k] += op->e[s] * vs[k];
      } else {
        axpy_g5(vs, -0.5, 0.5, y);
      }
    }
  }
}

/* U^{-1}: afopr_Domainwall_eo-tmpl.h:1067-1119 */
static void U_inv(const oracle_dwf *op, double *v, const double *w)
{
  const int Ls = op->Ls;
  const double a = op->alpha;
#pragma omp parallel for schedule(static)
  for (int site = 0; site < op->Vh; ++site) {
    double y[NIN], t[NIN];
    double *vl = fld(op, v, site, Ls - 1);
    for (int k = 0; k < NIN; ++k) t[k] = 0;
    axpy_g5(t, 0.5 * (1 + a), 0.5 * (a - 1), cfld(op, w, site, Ls - 1));
    for (int k = 0; k < NIN; ++k) vl[k] = t[k] / (op->dp[Ls - 1] + op->g);
    for (int k = 0; k < NIN; ++k) y[k] = 0;
    axpy_g5(y, 0.5, 0.5, vl);
    for (int s = Ls - 2; s >= 0; --s) {
      double u[NIN];
      memcpy(u, cfld(op, w, site, s), NIN * sizeof(double));
      axpy_g5(u, 0.5 * op->dm[s], -0.5 * op->dm[s], fld(op, v, site, s + 1));
      for (int k = 0; k < NIN; ++k) u[k] = (u[k] - op->f[s] * y[k]) / op->dp[s];
      double *vs = fld(op, v, site, s);
      if (s == 0) {
        for (int k = 0; k < NIN; ++k) vs[k] = 0;
        axpy_g5(vs, 0.5 * (1 + a), 0.5 * (1 - a), u);
      } else {
        memcpy(vs, u, NIN * sizeof(double));
      }
    }
  }
}

/* U^{-dag}: afopr_Domainwall_eo-tmpl.h:1124-1192 */
static void Udag_inv(const oracle_dwf *op, double *v, const double *w)
{
  const int Ls = op->Ls;
  const double a = op->alpha;
#pragma omp parallel for schedule(static)
  for (int site = 0; site < op->Vh; ++site) {
    double y[NIN], t[NIN];
    double *v0 = fld(op, v, site, 0);
    for (int k = 0; k < NIN; ++k) t[k] = 0;
    axpy_g5(t, 0.5 * (1 + a), 0.5 * (1 - a), cfld(op, w, site, 0));
    for (int k = 0; k < NIN; ++k) v0[k] = t[k] / op->dp[0];
    for (int k = 0; k < NIN; ++k) y[k] = op->f[0] * v0[k];
    for (int s = 1; s < Ls; ++s) {
      double u[NIN];
      memcpy(u, cfld(op, w, site, s), NIN * sizeof(double));
      axpy_g5(u, 0.5 * op->dm[s - 1], -0.5 * op->dm[s - 1], fld(op, v, site, s - 1));
      double *vs = fld(op, v, site, s);
      if (s < Ls - 1) {
        for (int k = 0; k < NIN; ++k) vs[k] = u[k] / op->dp[s];
        for (int k = 0; k < NIN; ++k) y[k] += op->f[s] * vs[k];
      } else {
        axpy_g5(u, -0.5, -0.5, y);
        for (int k = 0; k < NIN; ++k) u[k] /= (op->dp[Ls - 1] + op->g);
        for (int k = 0; k < NIN; ++k) vs[k] = 0;
        axpy_g5(vs, 0.5 * (1 + a), 0.5 * (a - 1), u);
      }
    }
  }
}

/* L^{-dag}: afopr_Domainwall_eo-tmpl.h:1197-1240 */
static void Ldag_inv(const oracle_dwf *op, double *v, const double *w)
{
  const int Ls = op->Ls;
#pragma omp parallel for schedule(static)
  for (int site = 0; site < op->Vh; ++site) {
    double y[NIN];
    memcpy(fld(op, v, site, Ls - 1), cfld(op, w, site, Ls - 1), NIN * sizeof(double));
    for (int k = 0; k < NIN; ++k) y[k] = 0;
    axpy_g5(y, 0.5, -0.5, cfld(op, w, site, Ls - 1));
    for (int s = Ls - 2; s >= 0; --s) {
      double t[NIN];
      double a = 0.5 * op->dm[s + 1] / op->dp[s];
      for (int k = 0; k < NIN; ++k) t[k] = 0;
      axpy_g5(t, a, a, fld(op, v, site, s + 1));
      double *vs = fld(op, v, site, s);
      const double *ws = cfld(op, w, site, s);
      for (int k = 0; k < NIN; ++k) vs[k] = ws[k] + (t[k] - op->e[s] * y[k]);
    }
  }
}

static void LU_inv(oracle_dwf *op, double *v, const double *w)
{
  L_inv(op, op->w3, w);
  U_inv(op, v, op->w3);
}

static void LUdag_inv(oracle_dwf *op, double *v, const double *w)
{
  Udag_inv(op, op->w3, w);
  Ldag_inv(op, v, op->w3);
}

static void gm5R(const oracle_dwf *op, double *v, const double *w)
{
  for (int s = 0; s < op->Ls; ++s)
    for (int site = 0; site < op->Vh; ++site)
      gamma_mult(fld(op, v, site, op->Ls - 1 - s), cfld(op, w, site, s), 4);
}

static void Rrefl(const oracle_dwf *op, double *v, const double *w)
{
  for (int s = 0; s < op->Ls; ++s)
    memcpy(fld(op, v, 0, op->Ls - 1 - s), cfld(op, w, 0, s),
           (size_t)NIN * op->Vh * sizeof(double));
}

/* D = 1 - M_ee^-1 D_eo M_oo^-1 D_oe  (afopr_Domainwall_eo-tmpl.h:652-665) */
static void Dfull(oracle_dwf *op, double *v, const double *w)
{
  size_t n = (size_t)NIN * op->Vh * op->Ls;
  D_eo(op, op->w1, w, 1);
  LU_inv(op, op->w2, op->w1);
  D_eo(op, op->w1, op->w2, 0);
  LU_inv(op, op->w2, op->w1);
  for (size_t i = 0; i < n; ++i) v[i] = w[i] - op->w2[i];
}

/* D^+ (afopr_Domainwall_eo-tmpl.h:690-707) */
static void Ddag(oracle_dwf *op, double *v, const double *w)
{
  size_t n = (size_t)NIN * op->Vh * op->Ls;
  LUdag_inv(op, op->w1, w);
  Ddag_eo(op, op->w2, op->w1, 1);
  LUdag_inv(op, op->w1, op->w2);
  Ddag_eo(op, op->w2, op->w1, 0);
  for (size_t i = 0; i < n; ++i) v[i] = w[i] - op->w2[i];
}

int oracle_dwf_mult(oracle_dwf *op, const char *mode, int dag, double *out,
                    const double *in)
{
  size_t n = (size_t)NIN * op->Vh * op->Ls;
  if (!strcmp(mode, "Deo")) {
    if (dag) Ddag_eo(op, out, in, 1); else D_eo(op, out, in, 0);
  } else if (!strcmp(mode, "Doe")) {
    if (dag) Ddag_eo(op, out, in, 0); else D_eo(op, out, in, 1);
  } else if (!strcmp(mode, "Dee") || !strcmp(mode, "Doo")) {
    D_ee(op, out, in, dag);
  } else if (!strcmp(mode, "Dee_inv") || !strcmp(mode, "Doo_inv")) {
    if (dag) LUdag_inv(op, out, in); else LU_inv(op, out, in);
  } else if (!strcmp(mode, "D")) {
    if (dag) Ddag(op, out, in); else Dfull(op, out, in);
  } else if (!strcmp(mode, "Ddag")) {
    if (dag) Dfull(op, out, in); else Ddag(op, out, in);
  } else if (!strcmp(mode, "DdagD")) {
    double *t = (double *)malloc(n * sizeof(double));
    Dfull(op, t, in);
    Ddag(op, out, t);
    free(t);
  } else if (!strcmp(mode, "H")) {
    /* H = gm5R D;  H^+ = D^+ gm5R  (afopr_Domainwall_eo-tmpl.h:669-686, 711-731) */
    double *t = (double *)malloc(n * sizeof(double));
    if (dag) { gm5R(op, t, in); Ddag(op, out, t); }
    else { Dfull(op, t, in); gm5R(op, out, t); }
    free(t);
  } else if (!strcmp(mode, "Hdag")) {
    double *t = (double *)malloc(n * sizeof(double));
    if (!dag) { gm5R(op, t, in); Ddag(op, out, t); }
    else { Dfull(op, t, in); gm5R(op, out, t); }
    free(t);
  } else if (!strcmp(mode, "gm5R")) {
    gm5R(op, out, in);
  } else if (!strcmp(mode, "R")) {
    Rrefl(op, out, in);
  } else {
    return -1;
  }
  return 0;
}

/* ---------------- solvers ---------------- */

static double dotr(size_t n, const double *a, const double *b)
{
  double s = 0;
  for (size_t i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}

static void apply_DdagD(oracle_dwf *op, double *out, const double *in, double *tmp)
{
  Dfull(op, tmp, in);
  Ddag(op, out, tmp);
}

/* reference src/lib_alt/Solver/asolver_CG-tmpl.h:118-234 (ZERO init guess) */
int oracle_cg(oracle_dwf *op, double *x, const double *b, double tol2,
              int maxiter, int *nconv, double *diff)
{
  size_t n = (size_t)NIN * op->Vh * op->Ls;
  double *r = (double *)malloc(n * sizeof(double));
  double *p = (double *)malloc(n * sizeof(double));
  double *s = (double *)malloc(n * sizeof(double));
  double *tmp = (double *)malloc(n * sizeof(double));
  double snorm = 1.0 / dotr(n, b, b);
  memcpy(r, b, n * sizeof(double));
  memcpy(p, b, n * sizeof(double));
  memset(x, 0, n * sizeof(double));
  double rr = dotr(n, r, r), rrp = rr;
  int conv = -1;
  for (int it = 0; it < maxiter; ++it) {
    apply_DdagD(op, s, p, tmp);
    double pap = dotr(n, s, p);
    double cr = rrp / pap;
    for (size_t i = 0; i < n; ++i) x[i] += cr * p[i];
    for (size_t i = 0; i < n; ++i) r[i] -= cr * s[i];
    rr = dotr(n, r, r);
    double bk = rr / rrp;
    for (size_t i = 0; i < n; ++i) p[i] = r[i] + bk * p[i];
    rrp = rr;
    if (rr * snorm < tol2) { conv = it + 1; break; }
  }
  apply_DdagD(op, s, x, tmp);
  for (size_t i = 0; i < n; ++i) s[i] -= b[i];
  if (diff) *diff = sqrt(dotr(n, s, s) * snorm);
  if (nconv) *nconv = conv;
  free(r); free(p); free(s); free(tmp);
  return conv < 0 ? 1 : 0;
}

/* reference src/lib/Solver/ashiftsolver_CG-tmpl.h:89-329 */
int oracle_shiftcg(oracle_dwf *op, double *x, const double *sigma, int nshift,
                   const double *b, double tol2, int maxiter, int *nconv,
                   double *diff)
{
  size_t n = (size_t)NIN * op->Vh * op->Ls;
  double *r = (double *)malloc(n * sizeof(double));
  double *s = (double *)malloc(n * sizeof(double));
  double *tmp = (double *)malloc(n * sizeof(double));
  double *p = (double *)malloc(n * nshift * sizeof(double));
  double *zeta1 = (double *)malloc(nshift * sizeof(double));
  double *zeta2 = (double *)malloc(nshift * sizeof(double));
  double *csh2 = (double *)malloc(nshift * sizeof(double));
  double *pp = (double *)malloc(nshift * sizeof(double));
  double snorm = 1.0 / dotr(n, b, b);
  for (int i = 0; i < nshift; ++i) {
    memcpy(p + n * i, b, n * sizeof(double));
    memset(x + n * i, 0, n * sizeof(double));
    zeta1[i] = zeta2[i] = 1.0;
    csh2[i] = sigma[i] - sigma[0];
    pp[i] = 0.0;
  }
  memcpy(r, b, n * sizeof(double));
  double rr = dotr(n, r, r);
  double alpha_p = 0.0, beta_p = 1.0;
  int nact = nshift;
  int conv = -1;
  for (int it = 0; it < maxiter; ++it) {
    apply_DdagD(op, s, p, tmp);
    for (size_t i = 0; i < n; ++i) s[i] += sigma[0] * p[i];
    double rr_p = rr;
    double pa_p = dotr(n, s, p);
    double beta = -rr_p / pa_p;
    for (size_t i = 0; i < n; ++i) x[i] -= beta * p[i];
    for (size_t i = 0; i < n; ++i) r[i] += beta * s[i];
    rr = dotr(n, r, r);
    double alpha = rr / rr_p;
    for (size_t i = 0; i < n; ++i) p[i] = r[i] + alpha * p[i];
    pp[0] = rr;
    double alpha_h = 1.0 + alpha_p * beta / beta_p;
    for (int ish = 1; ish < nact; ++ish) {
      double zeta = (alpha_h - csh2[ish] * beta) / zeta1[ish] + (1.0 - alpha_h) / zeta2[ish];
      zeta = 1.0 / zeta;
      double zr = zeta / zeta1[ish];
      double beta_s = beta * zr;
      double alpha_s = alpha * zr * zr;
      double *xi = x + n * ish, *pi = p + n * ish;
      for (size_t i = 0; i < n; ++i) xi[i] -= beta_s * pi[i];
      for (size_t i = 0; i < n; ++i) pi[i] = alpha_s * pi[i] + zeta * r[i];
      pp[ish] = dotr(n, pi, pi) * snorm;
      zeta2[ish] = zeta1[ish];
      zeta1[ish] = zeta;
    }
    int ish1 = nact;
    for (int ish = nact - 1; ish >= 0; --ish) {
      if (pp[ish] > tol2) { ish1 = ish + 1; break; }
    }
    nact = ish1;
    alpha_p = alpha;
    beta_p = beta;
    if (rr * snorm < tol2) { conv = it + 1; break; }
  }
  double dmax = 0.0;
  for (int i = 0; i < nshift; ++i) {
    apply_DdagD(op, s, x + n * i, tmp);
    for (size_t k = 0; k < n; ++k) s[k] += sigma[i] * x[n * i + k] - b[k];
    double d = sqrt(dotr(n, s, s) * snorm);
    if (d > dmax) dmax = d;
  }
  if (diff) *diff = dmax;
  if (nconv) *nconv = conv;
  free(r); free(s); free(tmp); free(p); free(zeta1); free(zeta2); free(csh2); free(pp);
  return conv < 0 ? 1 : 0;
}


/* ---------------- fermion force ---------------- */

/* Forward-mu part of the Wilson hop, output parity ieo:
 * out(x) = ph * (1 - g_mu) U_mu(x) in(x+mu)   (Fopr_Wilson_eo::mult_up,
 * src/lib/Fopr/Imp/fopr_Wilson_eo_impl.cpp:656-677) */
static void hop_up(const oracle_dwf *op, double *out, const double *in, int ieo, int mu)
{
  const int *L = op->L;
  const int Ls = op->Ls;
  for (int site = 0; site < op->Vh; ++site) {
    int ix2 = site % op->Nx2;
    int iyzt = site / op->Nx2;
    int y = iyzt % L[1];
    int z = (iyzt / L[1]) % L[2];
    int t = iyzt / (L[1] * L[2]);
    int keo = (ieo + y + z + t) % 2;
    int nc[4] = {2 * ix2 + keo, y, z, t};
    double ph = 1.0;
    if (nc[mu] == L[mu] - 1) { nc[mu] = 0; ph = op->bc[mu]; } else nc[mu] += 1;
    int nb = nc[0] / 2 + op->Nx2 * (nc[1] + L[1] * (nc[2] + L[2] * nc[3]));
    const double *u = op->ueo + (size_t)NDF * (site + (size_t)op->Vh * (ieo + 2 * mu));
    for (int s = 0; s < Ls; ++s) {
      const double *w = cfld(op, in, nb, s);
      double tmp[NIN], gt[NIN];
      for (int sp = 0; sp < NSP; ++sp) su3_mult(tmp + 6 * sp, u, w + 6 * sp);
      gamma_mult(gt, tmp, mu);
      double *o = fld(op, out, site, s);
      for (int k = 0; k < NIN; ++k) o[k] = ph * (tmp[k] - gt[k]);
    }
  }
}

/* AFopr_Domainwall_eo::mult_up (afopr_Domainwall_eo-tmpl.h:1262-1316):
 * the forward-mu part of D_eo, -1/2 hop_up(b w + c V(w)) (alpha = 1) */
static void mult_up(oracle_dwf *op, double *out, const double *w, int ieo, int mu)
{
  size_t n = (size_t)NIN * op->Vh * op->Ls;
  m5_apply(op, op->w4, w, op->b, op->c);
  hop_up(op, out, op->w4, ieo, mu);
  for (size_t i = 0; i < n; ++i) out[i] *= -0.5;
}

/* AFopr_Domainwall_eo::mult_up_dag (afopr_Domainwall_eo-tmpl.h:1376-1420):
 * M5^+ applied to -1/2 g5 hop_up(g5 w) */
static void mult_up_dag(oracle_dwf *op, double *out, const double *w, int ieo, int mu)
{
  size_t n = (size_t)NIN * op->Vh * op->Ls;
  g5_field(op, out, w);
  hop_up(op, op->w4, out, ieo, mu);
  g5_field(op, out, op->w4);
  for (size_t i = 0; i < n; ++i) out[i] *= -0.5;
  memcpy(op->w4, out, n * sizeof(double));
  m5_apply_dag(op, out, op->w4, op->b, op->c);
}

/* force_eo[mu](x) += sum_s sum_spin (U^+ work)(x)_c1 conj(v(x)_c2)
 * (mult_Field_Gd + tensorProd_Field_F, src/lib/Force/Fermion/Imp/tensorProd.cpp:39-98),
 * written into the lexical force for the sites of parity ieo */
static void accumulate_force(const oracle_dwf *op, double *force_lex, const double *v,
                             const double *work, int ieo, int mu)
{
  const int *L = op->L;
  for (int site = 0; site < op->Vh; ++site) {
    int ix2 = site % op->Nx2;
    int iyzt = site / op->Nx2;
    int y = iyzt % L[1];
    int z = (iyzt / L[1]) % L[2];
    int t = iyzt / (L[1] * L[2]);
    int x = 2 * ix2 + (ieo + y + z + t) % 2;
    int lex = x + L[0] * (y + L[1] * (z + L[2] * t));
    const double *u = op->ueo + (size_t)NDF * (site + (size_t)op->Vh * (ieo + 2 * mu));
    double *F = force_lex + (size_t)NDF * (lex + (size_t)op->V * mu);
    for (int s = 0; s < op->Ls; ++s) {
      const double *wk = cfld(op, work, site, s);
      const double *vv = cfld(op, v, site, s);
      double w2[NIN];
      for (int sp = 0; sp < NSP; ++sp) su3_dag_mult(w2 + 6 * sp, u, wk + 6 * sp);
      for (int c1 = 0; c1 < NC; ++c1)
        for (int c2 = 0; c2 < NC; ++c2)
          for (int sp = 0; sp < NSP; ++sp) {
            double ar = w2[2 * (c1 + 3 * sp)], ai = w2[2 * (c1 + 3 * sp) + 1];
            double br = vv[2 * (c2 + 3 * sp)], bi = vv[2 * (c2 + 3 * sp) + 1];
            F[2 * (c2 + 3 * c1)] += ar * br + ai * bi;
            F[2 * (c2 + 3 * c1) + 1] += ai * br - ar * bi;
          }
    }
  }
}

int oracle_dwf_force_udiv1(oracle_dwf *op, const char *mode, double *force_lex,
                           const double *a, const double *b)
{
  size_t n = (size_t)NIN * op->Vh * op->Ls;
  size_t nf = (size_t)NDF * op->V * 4;
  double *ue = (double *)malloc(n * sizeof(double));
  double *uo = (double *)malloc(n * sizeof(double));
  double *ve = (double *)malloc(n * sizeof(double));
  double *vo = (double *)malloc(n * sizeof(double));
  double *work = (double *)malloc(n * sizeof(double));
  double *work2 = (double *)malloc(n * sizeof(double));
  int hdag;
  if (!strcmp(mode, "H")) hdag = 0;
  else if (!strcmp(mode, "Hdag")) hdag = 1;
  else { free(ue); free(uo); free(ve); free(vo); free(work); free(work2); return -1; }
  memset(force_lex, 0, nf * sizeof(double));
  if (!hdag) {
    /* H: a = zeta_e, b = eta_e  (force_F_Domainwall_eo.cpp:190-247) */
    memcpy(ue, b, n * sizeof(double));
    D_eo(op, work, ue, 1);
    LU_inv(op, uo, work);
    gm5R(op, work, a);
    LUdag_inv(op, ve, work);
    Ddag_eo(op, work, ve, 1);
    LUdag_inv(op, vo, work);
    for (int mu = 0; mu < 4; ++mu) {
      mult_up(op, work2, uo, 0, mu);
      accumulate_force(op, force_lex, ve, work2, 0, mu);
    }
    for (int mu = 0; mu < 4; ++mu) {
      mult_up(op, work2, ue, 1, mu);
      accumulate_force(op, force_lex, vo, work2, 1, mu);
    }
  } else {
    /* Hdag: a = eta_e, b = zeta_e  (force_F_Domainwall_eo.cpp:251-318) */
    memcpy(ve, a, n * sizeof(double));
    D_eo(op, work, ve, 1);
    LU_inv(op, vo, work);
    gm5R(op, work, b);
    LUdag_inv(op, ue, work);
    Ddag_eo(op, work, ue, 1);
    LUdag_inv(op, uo, work);
    for (int mu = 0; mu < 4; ++mu) {
      mult_up_dag(op, work2, uo, 0, mu);
      accumulate_force(op, force_lex, ve, work2, 0, mu);
    }
    for (int mu = 0; mu < 4; ++mu) {
      mult_up_dag(op, work2, ue, 1, mu);
      accumulate_force(op, force_lex, vo, work2, 1, mu);
    }
  }
  for (size_t i = 0; i < nf; ++i) force_lex[i] = -force_lex[i];
  free(ue); free(uo); free(ve); free(vo); free(work); free(work2);
  return 0;
}

int oracle_dwf_force_udiv(oracle_dwf *op, double *force_lex, const double *eta)
{
  size_t n = (size_t)NIN * op->Vh * op->Ls;
  size_t nf = (size_t)NDF * op->V * 4;
  double *zeta = (double *)malloc(n * sizeof(double));
  double *f2 = (double *)malloc(nf * sizeof(double));
  oracle_dwf_mult(op, "H", 0, zeta, eta);
  oracle_dwf_force_udiv1(op, "H", force_lex, zeta, eta);
  oracle_dwf_force_udiv1(op, "Hdag", f2, eta, zeta);
  for (size_t i = 0; i < nf; ++i) force_lex[i] += f2[i];
  free(zeta);
  free(f2);
  return 0;
}
