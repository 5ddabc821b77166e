// AFopr_Domainwall_5din_eo<AField<REAL, B200>>: the reference's even/odd 5D
// domain-wall operator interface (src/lib_alt_Accel/Fopr/
// afopr_Domainwall_5din_eo.h:40-232, parameters as in -tmpl.h:246-299) with
// every mode run by the B200 library (b200_dwf_*), registered in the
// reference's factory under the same name, "Domainwall_5din_eo", so that
// AFopr<AField<REAL, B200>>::New("Domainwall_5din_eo", params) inside the
// reference's solver and action templates builds it.
//
// Fields are AField<REAL, B200> of nin = 24*Ls, nvol = Nvol/2, nex = 1 holding
// the library's device layout; convert / reverse move the reference's host
// Field(24, Nvol/2, Ls) in and out.  Calls come from inside the templates'
// OpenMP regions: thread 0 launches, barriers order the threads (the
// reference's ith_kernel pattern, -tmpl.h:979-1101).
#ifndef B200_AFOPR_DOMAINWALL_5DIN_EO_INCLUDED
#define B200_AFOPR_DOMAINWALL_5DIN_EO_INCLUDED

#include <string>
#include <vector>

#include "lib/Fopr/afopr.h"
#include "lib/Parameters/commonParameters.h"
#include "lib/Parameters/parameters.h"
#include "lib_alt_B200/Field/afield.h"

template<typename AFIELD> class AFopr_Domainwall_5din_eo;

template<typename REALTYPE>
class AFopr_Domainwall_5din_eo<AField<REALTYPE, B200> > : public AFopr<AField<REALTYPE, B200> >
{
 public:
  typedef AField<REALTYPE, B200> AFIELD;
  typedef REALTYPE real_t;
  static const std::string class_name;

 private:
  b200_dwf_t *m_op = nullptr;
  std::string m_mode = "D";
  int m_Ns = 0;
  int m_nvol2 = 0;
  AFIELD m_t;   // work field of mult_gm5

 public:
  AFopr_Domainwall_5din_eo(const Parameters& params) : AFopr<AFIELD>() { set_parameters(params); }
  ~AFopr_Domainwall_5din_eo() { if (m_op) b200_dwf_destroy(m_op); }

  void set_parameters(const Parameters& params)
  {
    std::string repr = "Dirac";
    params.fetch_string("gamma_matrix_type", repr);
    if (repr != "Dirac") {
      Bridge::vout.crucial("%s: gamma_matrix_type %s is not supported (Dirac only, as the Accel "
                           "operator)\n", class_name.c_str(), repr.c_str());
      exit(EXIT_FAILURE);
    }
    double mq, M0;
    int Ns;
    std::vector<int> bc;
    int err = 0;
    err += params.fetch_double("quark_mass", mq);
    err += params.fetch_double("domain_wall_height", M0);
    err += params.fetch_int("extent_of_5th_dimension", Ns);
    err += params.fetch_int_vector("boundary_condition", bc);
    if (err || bc.size() != 4) {
      Bridge::vout.crucial("Error at %s: input parameter not found.\n", class_name.c_str());
      exit(EXIT_FAILURE);
    }
    double b = 1.0, c = 0.0, alpha = 1.0;
    if (params.fetch_double("coefficient_b", b) + params.fetch_double("coefficient_c", c)) {
      b = 1.0;
      c = 0.0;
    }
    if (params.fetch_double("parameter_alpha", alpha)) alpha = 1.0;
    const int lat[4] = {CommonParameters::Nx(), CommonParameters::Ny(), CommonParameters::Nz(),
                        CommonParameters::Nt()};
    std::vector<double> bs(Ns, b), cs(Ns, c);
    if (m_op) b200_dwf_destroy(m_op);
    m_op = nullptr;
    b200_overlay::check(b200_dwf_create(&m_op, lat, Ns, mq, M0, bs.data(), cs.data(), alpha, bc.data()),
                        "AFopr_Domainwall_5din_eo<B200>::set_parameters");
    m_Ns = Ns;
    m_nvol2 = CommonParameters::Nvol() / 2;
  }

  void set_config(Field *U)
  {
    if (ThreadManager::get_thread_id() == 0)
      b200_overlay::check(b200_dwf_set_config(m_op, U->ptr(0), nullptr), "set_config");
#pragma omp barrier
  }

  void set_mode(std::string mode) { m_mode = mode; }
  std::string get_mode() const { return m_mode; }

  void mult(AFIELD& v, const AFIELD& w) { apply(v, w, m_mode, 0); }
  void mult_dag(AFIELD& v, const AFIELD& w) { apply(v, w, m_mode, 1); }
  void mult(AFIELD& v, const AFIELD& w, const std::string mode) { apply(v, w, mode, 0); }
  void mult_dag(AFIELD& v, const AFIELD& w, const std::string mode) { apply(v, w, mode, 1); }

  // gamma_5 = (gamma_5 R) R on the 5D field
  void mult_gm5(AFIELD& v, const AFIELD& w)
  {
    if (!m_t.check_size(w)) m_t.reset(w.nin(), w.nvol(), w.nex());
    apply(m_t, w, "R", 0);
    apply(v, m_t, "gm5R", 0);
  }

  int field_nin() { return 24 * m_Ns; }
  int field_nvol() { return m_nvol2; }
  int field_nex() { return 1; }
  bool needs_convert() { return true; }

  // host Field(24, Nvol/2, Ls) in the reference's layout <-> device field
  void convert(AFIELD& v, const Field& w)
  {
    if (ThreadManager::get_thread_id() == 0)
      b200_overlay::check(b200_field_convert(m_op, AFIELD::prec(), v.ptr(0), w.ptr(0), nullptr), "convert");
#pragma omp barrier
  }
  void reverse(Field& v, const AFIELD& w)
  {
    if (ThreadManager::get_thread_id() == 0)
      b200_overlay::check(b200_field_reverse(m_op, AFIELD::prec(), v.ptr(0), w.ptr(0), nullptr), "reverse");
#pragma omp barrier
  }

  // the fused hop's algorithmic flops (1488*Ls per half-site and D_eo,
  // afopr_Domainwall_5din_eo-tmpl.h:1445-1492) times the hops of the mode
  double flop_count() { return flop_count(m_mode); }
  double flop_count(const std::string mode)
  {
    const double hop = 1488.0 * m_Ns * double(m_nvol2);
    if (mode == "Deo" || mode == "Doe") return hop;
    if (mode == "D" || mode == "Ddag" || mode == "H" || mode == "Hdag") return 2.0 * hop;
    if (mode == "DdagD") return 4.0 * hop;
    return 0.0;
  }

  b200_dwf_t *handle() { return m_op; }

 private:
  void apply(AFIELD& v, const AFIELD& w, const std::string& mode, int dag)
  {
    if (ThreadManager::get_thread_id() == 0)
      b200_overlay::check(b200_dwf_mult(m_op, AFIELD::prec(), v.ptr(0), w.ptr(0), mode.c_str(), dag, nullptr),
                          "AFopr_Domainwall_5din_eo<B200>::mult");
#pragma omp barrier
  }

#ifdef USE_FACTORY
  static AFopr<AFIELD> *create_object_with_params(const Parameters& params)
  { return new AFopr_Domainwall_5din_eo(params); }

 public:
  static bool register_factory()
  {
    return AFopr<AFIELD>::Factory_params::Register("Domainwall_5din_eo", create_object_with_params);
  }
#endif
};

template<typename REALTYPE>
const std::string AFopr_Domainwall_5din_eo<AField<REALTYPE, B200> >::class_name
  = "AFopr_Domainwall_5din_eo<AField<REAL,B200> >";

#endif
