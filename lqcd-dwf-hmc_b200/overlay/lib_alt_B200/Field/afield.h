// AField<REAL, B200>: the reference's alt field container with its data on
// the B200, for the reference's own solver templates (ASolver_CG,
// ASolver_Richardson, APrecond_Mixedprec, AShiftsolver_CG,
// Fprop_alt_Standard_eo_Richardson) running over the B200 domain-wall operator.
//
// Interface: the reference's AField<REAL, ACCEL> (src/lib_alt_Accel/Field/
// afield.h:30-240) as far as those templates use it; the data is one device
// array of nin*nvol*nex reals that the library's operator reads in its own
// site-major layout (nin = 24*Ls, nvol = Nvol/2, nex = 1 for a 5D half-lattice
// spinor).  Vector work runs in the library's flat kernels (b200_blas_*).
// Threading follows the reference: the templates call these methods from every
// OpenMP thread; thread 0 launches, a barrier orders the threads, and a
// reduction's value is handed to all threads by ThreadManager::reduce_sum_global
// (afield-tmpl.h's norm2 pattern).  The containers hold no host mirror:
// update_host / update_device are no-ops.
#ifndef B200_AFIELD_INCLUDED
#define B200_AFIELD_INCLUDED

#include <cassert>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <string>

#include <cuda_runtime.h>

#include "lib_alt/Field/afield_base.h"
#include "bridge_defs.h"
#include "bridge_complex.h"
#include "complexTraits.h"
#include "lib/Field/field.h"
#include "lib/IO/bridgeIO.h"
#include "lib/ResourceManager/threadManager.h"

#include "b200dwf.h"

namespace b200_overlay {
// The library's status as the reference reports misuse: vout.crucial + exit.
inline void check(int rc, const char* what)
{
  if (rc != 0) {
    Bridge::vout.crucial("%s: %s\n", what, b200_last_error());
    exit(EXIT_FAILURE);
  }
}

template<typename R> struct Prec;
template<> struct Prec<double> { static const int v = 0; };
template<> struct Prec<float>  { static const int v = 1; };
}  // namespace b200_overlay

template<typename REALTYPE>
class AField<REALTYPE, B200>
{
 public:
  typedef REALTYPE real_t;
  typedef typename ComplexTraits<REALTYPE>::complex_t complex_t;
  typedef Element_type::type element_type;

  static const Impl IMPL = B200;
  static const std::string class_name;

 protected:
  int m_nin, m_nvol, m_nex;
  element_type m_element_type;
  std::size_t m_nsize;
  real_t *m_field;   // device

 public:
  AField() : m_nin(0), m_nvol(0), m_nex(0), m_element_type(Element_type::COMPLEX), m_nsize(0),
             m_field(nullptr) {}

  AField(const int nin, const int nvol, const int nex,
         const element_type cmpl = Element_type::COMPLEX)
    : m_nin(0), m_nvol(0), m_nex(0), m_element_type(cmpl), m_nsize(0), m_field(nullptr)
  { reset(nin, nvol, nex, cmpl); }

  AField(const AField& w)
    : m_nin(0), m_nvol(0), m_nex(0), m_element_type(w.m_element_type), m_nsize(0), m_field(nullptr)
  {
    reset(w.nin(), w.nvol(), w.nex(), w.field_element_type());
    if (m_nsize > 0) copy(w);
  }

  AField& operator=(const AField& w)
  {
    assert(check_size(w));
    if (m_nsize > 0) copy(w);
    return *this;
  }

  ~AField() { release(); }

  void reset(const int nin, const int nvol, const int nex,
             const element_type cmpl = Element_type::COMPLEX)
  {
    const std::size_t n = std::size_t(nin) * nvol * nex;
    m_element_type = cmpl;
    if (n == m_nsize && m_field) { m_nin = nin; m_nvol = nvol; m_nex = nex; return; }
    int ith = ThreadManager::get_thread_id();
#pragma omp barrier
    if (ith == 0) {
      release();
      m_nin = nin; m_nvol = nvol; m_nex = nex; m_nsize = n;
      if (n > 0 && cudaMalloc(&m_field, n * sizeof(real_t)) != cudaSuccess) {
        Bridge::vout.crucial("AField<B200>: cudaMalloc of %zu reals failed\n", n);
        exit(EXIT_FAILURE);
      }
      if (n > 0) b200_overlay::check(b200_blas_fill(prec(), n, 0.0, m_field, nullptr), "AField::reset");
    }
#pragma omp barrier
  }

  int nin() const { return m_nin; }
  int nvol() const { return m_nvol; }
  int nex() const { return m_nex; }
  element_type field_element_type() const { return m_element_type; }
  int size() const { return int(m_nsize); }
  bool check_size(const int nin, const int nvol, const int nex) const
  { return m_nin == nin && m_nvol == nvol && m_nex == nex; }
  bool check_size(const AField& w) const { return check_size(w.nin(), w.nvol(), w.nex()); }

  // device data, for the operator shell
  real_t *ptr(int i) { return m_field + i; }
  const real_t *ptr(int i) const { return m_field + i; }
  static int prec() { return b200_overlay::Prec<REALTYPE>::v; }

  void set(const real_t a)
  { on_thread0([&] { return b200_blas_fill(prec(), m_nsize, double(a), m_field, nullptr); }, "set"); }
  // one element (a point source): a host write into device memory
  void set(const int index, const real_t a)
  {
    assert(index >= 0 && std::size_t(index) < m_nsize);
    if (ThreadManager::get_thread_id() == 0)
      b200_overlay::check(cudaMemcpy(m_field + index, &a, sizeof(real_t), cudaMemcpyHostToDevice)
                          == cudaSuccess ? 0 : -2, "AField::set");
#pragma omp barrier
  }
  void copy(const AField& w)
  {
    assert(check_size(w));
    if (ThreadManager::get_thread_id() == 0 && w.m_field != m_field)
      b200_overlay::check(cudaMemcpy(m_field, w.m_field, m_nsize * sizeof(real_t), cudaMemcpyDeviceToDevice)
                          == cudaSuccess ? 0 : -2, "AField::copy");
#pragma omp barrier
  }
  // y = a w + y
  void axpy(const real_t a, const AField& w)
  {
    on_thread0([&] { return b200_blas_axpby(prec(), m_nsize, double(a), w.m_field, 1.0, m_field, nullptr); },
               "axpy");
  }
  void axpy(const complex_t a, const AField& w)
  {
    on_thread0([&] {
      return b200_blas_caxpby(prec(), m_nsize, double(real(a)), double(imag(a)), w.m_field, 1.0, 0.0,
                              m_field, nullptr);
    }, "axpy");
  }
  // y = a y + w
  void aypx(const real_t a, const AField& w)
  {
    on_thread0([&] { return b200_blas_axpby(prec(), m_nsize, 1.0, w.m_field, double(a), m_field, nullptr); },
               "aypx");
  }
  void aypx(const complex_t a, const AField& w)
  {
    on_thread0([&] {
      return b200_blas_caxpby(prec(), m_nsize, 1.0, 0.0, w.m_field, double(real(a)), double(imag(a)),
                              m_field, nullptr);
    }, "aypx");
  }
  void scal(const real_t a)
  {
    on_thread0([&] { return b200_blas_axpby(prec(), m_nsize, 0.0, nullptr, double(a), m_field, nullptr); },
               "scal");
  }
  void scal(const complex_t a)
  {
    on_thread0([&] {
      return b200_blas_caxpby(prec(), m_nsize, 0.0, 0.0, nullptr, double(real(a)), double(imag(a)),
                              m_field, nullptr);
    }, "scal");
  }
  real_t dot(const AField& w) const
  {
    double a = 0.0;
    if (ThreadManager::get_thread_id() == 0)
      b200_overlay::check(b200_blas_dot(prec(), m_nsize, m_field, w.m_field, &a, nullptr), "AField::dot");
    return share(a);
  }
  // <this, w> = sum conj(this) w
  void dotc(real_t& re, real_t& im, const AField& w) const
  {
    double r = 0.0, i = 0.0;
    if (ThreadManager::get_thread_id() == 0)
      b200_overlay::check(b200_blas_dotc(prec(), m_nsize, m_field, w.m_field, &r, &i, nullptr),
                          "AField::dotc");
    re = share(r);
    im = share(i);
  }
  real_t norm2() const { return dot(*this); }
  void update_host() const {}
  void update_device() {}

 private:
  void release()
  {
    if (m_field) cudaFree(m_field);
    m_field = nullptr;
    m_nsize = 0;
  }
  // the device work f() runs on thread 0 only; every thread waits for it
  template<typename F>
  void on_thread0(F f, const char* what)
  {
    if (ThreadManager::get_thread_id() == 0) b200_overlay::check(f(), what);
#pragma omp barrier
  }
  // thread 0 computed a; every thread returns it
  static real_t share(double a)
  {
    int ith = ThreadManager::get_thread_id(), nth = ThreadManager::get_num_threads();
    if (ith != 0) a = 0.0;
#pragma omp barrier
    ThreadManager::reduce_sum_global(a, ith, nth);
    return real_t(a);
  }
};

template<typename REALTYPE>
const std::string AField<REALTYPE, B200>::class_name = "AField<B200>";

// ------------------------------------------------------------ free functions
// (the reference's afield-inc.h forms the solver templates call)
template<typename R>
inline void copy(AField<R, B200>& v, const AField<R, B200>& w) { v.copy(w); }
template<typename R>
inline void axpy(AField<R, B200>& v, const R a, const AField<R, B200>& w) { v.axpy(a, w); }
template<typename R>
inline void axpy(AField<R, B200>& v, const typename ComplexTraits<R>::complex_t a,
                 const AField<R, B200>& w) { v.axpy(a, w); }
template<typename R>
inline void aypx(const R a, AField<R, B200>& v, const AField<R, B200>& w) { v.aypx(a, w); }
template<typename R>
inline void aypx(const typename ComplexTraits<R>::complex_t a, AField<R, B200>& v,
                 const AField<R, B200>& w) { v.aypx(a, w); }
template<typename R>
inline void scal(AField<R, B200>& v, const R a) { v.scal(a); }
template<typename R>
inline void scal(AField<R, B200>& v, const typename ComplexTraits<R>::complex_t a) { v.scal(a); }
template<typename R>
inline R dot(const AField<R, B200>& v, const AField<R, B200>& w) { return v.dot(w); }
template<typename R>
inline R norm2(const AField<R, B200>& v) { return v.norm2(); }
template<typename R>
inline typename ComplexTraits<R>::complex_t dotc(const AField<R, B200>& v, const AField<R, B200>& w)
{
  R re, im;
  v.dotc(re, im, w);
  return typename ComplexTraits<R>::complex_t(re, im);
}

// ------------------------------------------------------------ index tags
// The reference's AIndex_eo / AIndex_lex describe a field's site ordering
// per implementation (aindex_eo.h); here the order is the library's own and
// needs no state.  They select the precision conversions below.
template<typename REALTYPE, Impl IMPL> class AIndex_eo;
template<typename REALTYPE, Impl IMPL> class AIndex_lex;
// The B200 shell holds even/odd half-lattice fields only: the reference's
// full-lattice entry points (Fprop_alt::invert(Field&, ...), the index's
// split / merge, lexical Field <-> AField copies) stop with an error, as the
// reference does on unsupported use.
namespace b200_overlay {
inline void lexical_unsupported(const char* what)
{
  Bridge::vout.crucial("AField<B200>: %s on a full-lattice field is not provided "
                       "(the B200 shell works on even/odd half-lattice fields)\n", what);
  exit(EXIT_FAILURE);
}
}  // namespace b200_overlay

template<typename REALTYPE> class AIndex_eo<REALTYPE, B200>
{
 public:
  template<typename A> void split(A&, A&, const A&) { b200_overlay::lexical_unsupported("split"); }
  template<typename A> void merge(A&, const A&, const A&) { b200_overlay::lexical_unsupported("merge"); }
};
template<typename REALTYPE> class AIndex_lex<REALTYPE, B200> {};

template<typename R>
inline void convert(AIndex_lex<R, B200>&, AField<R, B200>&, const Field&)
{ b200_overlay::lexical_unsupported("convert"); }
template<typename R>
inline void reverse(AIndex_lex<R, B200>&, Field&, const AField<R, B200>&)
{ b200_overlay::lexical_unsupported("reverse"); }
template<typename R>
inline void convert_gauge(AIndex_lex<R, B200>&, AField<R, B200>&, const Field&)
{ b200_overlay::lexical_unsupported("convert_gauge"); }

// convert_h(index2, v2, index1, v1): the even/odd field v1 in the precision
// of v2 (APrecond_Mixedprec, src/lib_alt/Solver/aprecond_Mixedprec-tmpl.h:
// 73-104).  The storage layout differs between precisions, so the copy runs
// through the library's layout-aware conversion (nvol sites, Ls = nin / 24).
template<typename R2, typename R1>
inline void convert_h(AIndex_eo<R2, B200>&, AField<R2, B200>& v2,
                      AIndex_eo<R1, B200>&, const AField<R1, B200>& v1)
{
  assert(v2.check_size(v1));
  if (ThreadManager::get_thread_id() == 0)
    b200_overlay::check(b200_field_convert_prec(AField<R2, B200>::prec(), v2.ptr(0),
                                                AField<R1, B200>::prec(), v1.ptr(0), v1.nvol(),
                                                v1.nin() / 24, nullptr),
                        "convert_h");
#pragma omp barrier
}

// convert(index2, v2, index1, v1): the same precision copy for a field on
// the full lattice (APrecond_Mixedprec's LEXICAL branch); the library's
// layout is per site, so the copy is the same per-site conversion.
template<typename R2, typename R1>
inline void convert(AIndex_lex<R2, B200>&, AField<R2, B200>& v2,
                    AIndex_lex<R1, B200>&, const AField<R1, B200>& v1)
{
  assert(v2.check_size(v1));
  if (ThreadManager::get_thread_id() == 0)
    b200_overlay::check(b200_field_convert_prec(AField<R2, B200>::prec(), v2.ptr(0),
                                                AField<R1, B200>::prec(), v1.ptr(0), v1.nvol(),
                                                v1.nin() / 24, nullptr),
                        "convert");
#pragma omp barrier
}

#endif  // B200_AFIELD_INCLUDED
