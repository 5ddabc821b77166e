// b200dwf.hpp -- header-only C++ shells over the C ABI in b200dwf.h, shaped
// like the reference classes they stand in for, so that the reference's
// templates and driver can hold them where they hold the Accel ones:
//
//   AField_B200<REAL>         ~ AField<REAL, ACCEL>  (src/lib_alt_Accel/Field/afield.h)
//   AFopr_Domainwall_B200     ~ AFopr_Domainwall_5din_eo<AFIELD>
//                               (src/lib_alt_Accel/Fopr/afopr_Domainwall_5din_eo.h:40-232;
//                                virtual interface src/lib/Fopr/afopr.h:65-202)
//   ASolver_CG_B200           ~ ASolver_CG<AFIELD>::solve (src/lib_alt/Solver/asolver.h:51)
//   AShiftsolver_CG_B200      ~ AShiftsolver_CG<AFIELD>::solve (ashiftsolver_CG-tmpl.h:89-94)
//
// Error behaviour follows the reference at its interface: a failing call
// reports the library's message and terminates (the reference does
// vout.crucial + exit, afopr_Domainwall_5din_eo-tmpl.h:665-668); here the
// message goes to stderr and the handler is replaceable (b200::on_error).
// Device memory is owned by the fields (cudaMalloc/cudaFree via the CUDA
// runtime); nothing in these shells computes on the host.
#ifndef B200DWF_HPP
#define B200DWF_HPP

#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "b200dwf.h"

namespace b200 {

inline void (*&on_error())(const char*) {
  static void (*handler)(const char*) = nullptr;
  return handler;
}

inline void ok(int rc) {
  if (rc == 0) return;
  const char* msg = b200_last_error();
  if (on_error()) { on_error()(msg); return; }
  std::fprintf(stderr, "b200dwf: %s (code %d)\n", msg, rc);
  std::exit(EXIT_FAILURE);
}

template <typename REAL> struct PrecOf;
template <> struct PrecOf<double> { static constexpr int v = B200_F64; };
template <> struct PrecOf<float> { static constexpr int v = B200_F32; };

class AFopr_Domainwall_B200;

// One even/odd 5D half-lattice spinor in the library's device layout.
template <typename REAL>
class AField_B200 {
 public:
  typedef REAL real_t;
  AField_B200() = default;
  explicit AField_B200(AFopr_Domainwall_B200& op) { reset(op); }
  AField_B200(const AField_B200&) = delete;
  AField_B200& operator=(const AField_B200&) = delete;
  ~AField_B200() { if (m_dev) cudaFree(m_dev); }

  inline void reset(AFopr_Domainwall_B200& op);
  void* dev() { return m_dev; }
  const void* dev() const { return m_dev; }
  size_t bytes() const { return m_bytes; }
  b200_dwf_t* plan() const { return m_plan; }

  // AField BLAS (afield-tmpl.h:637-720)
  double norm2() const {
    double r = 0.0;
    ok(b200_field_norm2(m_plan, prec(), m_dev, &r, nullptr));
    return r;
  }
  double dot(const AField_B200& w) const {
    double r = 0.0;
    ok(b200_field_dot(m_plan, prec(), m_dev, w.m_dev, &r, nullptr));
    return r;
  }
  void axpy(double a, const AField_B200& x) { ok(b200_field_axpby(m_plan, prec(), m_dev, a, x.m_dev, 1.0, nullptr)); }
  void aypx(double a, const AField_B200& x) { ok(b200_field_axpby(m_plan, prec(), m_dev, 1.0, x.m_dev, a, nullptr)); }
  void scal(double a) { ok(b200_field_axpby(m_plan, prec(), m_dev, 0.0, nullptr, a, nullptr)); }
  void set(double a) {
    if (a != 0.0) { std::fprintf(stderr, "b200dwf: AField::set supports 0 only\n"); std::exit(EXIT_FAILURE); }
    ok(b200_field_axpby(m_plan, prec(), m_dev, 0.0, nullptr, 0.0, nullptr));
  }
  void copy(const AField_B200& x) { ok(b200_field_axpby(m_plan, prec(), m_dev, 1.0, x.m_dev, 0.0, nullptr)); }
  // convert_h between precisions (afield_copy_openacc-inc.h:11-54)
  template <typename R2>
  void convert_from(const AField_B200<R2>& x) {
    ok(b200_field_copy_convert(m_plan, prec(), m_dev, PrecOf<R2>::v, x.dev(), nullptr));
  }

 private:
  static constexpr int prec() { return PrecOf<REAL>::v; }
  b200_dwf_t* m_plan = nullptr;
  void* m_dev = nullptr;
  size_t m_bytes = 0;
};

class AFopr_Domainwall_B200 {
 public:
  // set_parameters (afopr_Domainwall_5din_eo-tmpl.h:246-301): Shamir when b, c are empty
  AFopr_Domainwall_B200(const int lattice[4], int Ls, double mq, double M0,
                        const std::vector<double>& b = {}, const std::vector<double>& c = {},
                        double alpha = 1.0, const std::vector<int>& bc = {1, 1, 1, -1})
      : m_ls(Ls), m_nvol(lattice[0] * lattice[1] * lattice[2] * lattice[3]) {
    ok(b200_dwf_create(&m_op, lattice, Ls, mq, M0, b.empty() ? nullptr : b.data(),
                       c.empty() ? nullptr : c.data(), alpha, bc.data()));
  }
  AFopr_Domainwall_B200(const AFopr_Domainwall_B200&) = delete;
  AFopr_Domainwall_B200& operator=(const AFopr_Domainwall_B200&) = delete;
  ~AFopr_Domainwall_B200() { b200_dwf_destroy(m_op); }

  b200_dwf_t* plan() { return m_op; }

  // AFopr virtual interface (afopr.h:65-202)
  void set_config(const double* u_lex_host) { ok(b200_dwf_set_config(m_op, u_lex_host, nullptr)); }
  void set_mode(const std::string& mode) { m_mode = mode; }
  std::string get_mode() const { return m_mode; }
  template <typename F> void mult(F& v, const F& w) { apply(v, w, m_mode, 0); }
  template <typename F> void mult_dag(F& v, const F& w) { apply(v, w, m_mode, 1); }
  template <typename F> void mult(F& v, const F& w, const std::string& mode) { apply(v, w, mode, 0); }
  template <typename F> void mult_dag(F& v, const F& w, const std::string& mode) { apply(v, w, mode, 1); }
  bool needs_convert() const { return true; }
  template <typename F> void convert(F& v, const double* w_host) {
    ok(b200_field_convert(m_op, PrecOf<typename F::real_t>::v, v.dev(), w_host, nullptr));
  }
  template <typename F> void reverse(double* v_host, const F& w) {
    ok(b200_field_reverse(m_op, PrecOf<typename F::real_t>::v, v_host, w.dev(), nullptr));
  }
  int field_nin() const { return 24 * m_ls; }
  int field_nvol() const { return m_nvol / 2; }
  int field_nex() const { return 1; }

 private:
  template <typename F>
  void apply(F& v, const F& w, const std::string& mode, int dag) {
    ok(b200_dwf_mult(m_op, PrecOf<typename F::real_t>::v, v.dev(), w.dev(), mode.c_str(), dag, nullptr));
  }
  b200_dwf_t* m_op = nullptr;
  std::string m_mode = "D";
  int m_ls, m_nvol;
};

template <typename REAL>
void AField_B200<REAL>::reset(AFopr_Domainwall_B200& op) {
  if (m_dev) cudaFree(m_dev);
  m_plan = op.plan();
  m_bytes = b200_dwf_field_bytes(m_plan, prec());
  if (cudaMalloc(&m_dev, m_bytes) != cudaSuccess) {
    std::fprintf(stderr, "b200dwf: cudaMalloc of %zu bytes failed\n", m_bytes);
    std::exit(EXIT_FAILURE);
  }
}

// ASolver_CG::solve(x, b, Nconv, diff) on DdagD (asolver_CG-tmpl.h:118-234)
template <typename REAL>
class ASolver_CG_B200 {
 public:
  ASolver_CG_B200(AFopr_Domainwall_B200& op, int niter, double stop_cond)
      : m_op(op), m_niter(niter), m_stop(stop_cond) {}
  void solve(AField_B200<REAL>& x, const AField_B200<REAL>& b, int& nconv, double& diff) {
    const int rc = b200_cg_solve(m_op.plan(), PrecOf<REAL>::v, x.dev(), b.dev(), m_niter, m_stop,
                                 &nconv, &diff, nullptr);
    if (rc != B200_ENOCONV) ok(rc);
  }

 private:
  AFopr_Domainwall_B200& m_op;
  int m_niter;
  double m_stop;
};

// AShiftsolver_CG::solve(xq, sigma, b, Nconv, diff) (ashiftsolver_CG-tmpl.h:89-94)
class AShiftsolver_CG_B200 {
 public:
  AShiftsolver_CG_B200(AFopr_Domainwall_B200& op, int niter, double stop_cond)
      : m_op(op), m_niter(niter), m_stop(stop_cond) {}
  void solve(std::vector<AField_B200<double>*>& xq, const std::vector<double>& sigma,
             const AField_B200<double>& b, int& nconv, double& diff) {
    std::vector<void*> x(xq.size());
    for (size_t i = 0; i < xq.size(); ++i) x[i] = xq[i]->dev();
    const int rc = b200_shiftcg_solve(m_op.plan(), x.data(), sigma.data(), (int)x.size(), b.dev(),
                                      m_niter, m_stop, &nconv, &diff, nullptr);
    if (rc != B200_ENOCONV) ok(rc);
    nconv -= 1;   // the reference reports iterations - 1
  }

 private:
  AFopr_Domainwall_B200& m_op;
  int m_niter;
  double m_stop;
};

}  // namespace b200

#endif
