// Harness that times the reference's own mixed-precision solver on the CPU:
// Fprop_alt_Standard_eo_Richardson<AField<double,QXS>, AField<float,QXS>>
// (src/lib_alt/Measurements/Fermion/fprop_alt_Standard_eo_Richardson-tmpl.h:
// 27-102, 460-481) over the reference's QXS operator
// AFopr_Domainwall_5din_eo<AField<REAL,QXS>> (src/lib_alt_QXS/Fopr/), both
// compiled from the reference's sources by oracle/Makefile.qxs.  The solver
// is the one the reference benchmark's ratio actions use
// (benchmark_hmc_dwf/hmc_dwf_eo.cpp:79, 311-324): FP64 Richardson outer
// iterations, each an FP32 CG on DdagD (APrecond_Mixedprec).
//
// This file is test / measurement infrastructure: nothing in the product
// links it.
//
// Usage:  qxs_harness <params.txt> <in_dir>
//   params.txt: "key value..." lines: lattice Nx Ny Nz Nt, Ls, mq, M0, b, c,
//   bc bx by bz bt, threads, reps (timed DdagD applications).
//   in_dir/gauge.bin, in_dir/src.bin: as for ref_harness (lexical
//   Field_G(Nvol, 4); even-site Field(24, Nvol/2, Ls)).
// Prints "key value" lines: the seconds of one FP64 and one FP32 DdagD of
// the QXS operator, and of one bounded solve (1 outer x 1 inner iteration).

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

// the Fprop's smeared-operator constructor needs the alt director's
// declaration, as the reference's own instantiation unit has it
#define DIRECTOR_ALT_SMEARED_IMPLEMENTED
#include "bridge_setup.h"
#include "lib/Parameters/commonParameters.h"
#include "lib/Parameters/parameters.h"
#include "lib/ResourceManager/threadManager.h"
#include "lib/Field/field.h"
#include "lib/Field/field_G.h"
#include "lib_alt/Smear/director_alt_Smear.h"
#include "lib_alt/Measurements/Fermion/fprop_alt_Standard_eo_Richardson.h"
#include "lib_alt_QXS/Field/afield.h"
#include "lib_alt_QXS/init_alt_QXS.h"

typedef AField<double, QXS> AFIELD_d;
typedef AField<float, QXS> AFIELD_f;

namespace {

typedef std::map<std::string, std::vector<std::string> > Kv;

Kv read_params(const char* path)
{
  Kv kv;
  std::ifstream f(path);
  std::string line;
  while (std::getline(f, line)) {
    std::istringstream is(line);
    std::string key;
    if (!(is >> key) || key[0] == '#') continue;
    std::vector<std::string> vals;
    std::string v;
    while (is >> v) vals.push_back(v);
    kv[key] = vals;
  }
  return kv;
}

double getd(const Kv& kv, const char* k, double def)
{
  Kv::const_iterator it = kv.find(k);
  return (it == kv.end() || it->second.empty()) ? def : atof(it->second[0].c_str());
}

int geti(const Kv& kv, const char* k, int def)
{
  Kv::const_iterator it = kv.find(k);
  return (it == kv.end() || it->second.empty()) ? def : atoi(it->second[0].c_str());
}

std::vector<int> getiv(const Kv& kv, const char* k)
{
  std::vector<int> r;
  Kv::const_iterator it = kv.find(k);
  if (it != kv.end())
    for (size_t i = 0; i < it->second.size(); ++i) r.push_back(atoi(it->second[i].c_str()));
  return r;
}

bool read_bin(const std::string& path, double* dst, size_t n)
{
  FILE* f = fopen(path.c_str(), "rb");
  if (!f) return false;
  const size_t got = fread(dst, sizeof(double), n, f);
  fclose(f);
  return got == n;
}

double now()
{
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// seconds of one mult in mode DdagD, averaged over reps, inside one
// OpenMP parallel region as the reference's mult_performance does
template <typename AF>
double time_ddagd(AFopr<AF>* fopr, int reps)
{
  const int nin = fopr->field_nin(), nvol = fopr->field_nvol(), nex = fopr->field_nex();
  AF y1(nin, nvol, nex), y2(nin, nvol, nex);
#pragma omp parallel
  {
    y1.set(0.0);
  }
  y1.set(0, 1.0);
  fopr->set_mode("DdagD");
#pragma omp parallel
  {
    fopr->mult(y2, y1);
  }
  const double t0 = now();
#pragma omp parallel
  {
    for (int i = 0; i < reps; ++i) {
      fopr->mult(y2, y1);
      fopr->mult(y1, y2);
    }
  }
  return (now() - t0) / (2.0 * reps);
}

}  // namespace

int main(int argc, char** argv)
{
  if (argc < 3) {
    fprintf(stderr, "usage: %s params.txt in_dir\n", argv[0]);
    return 2;
  }
  Kv kv = read_params(argv[1]);
  const std::string in_dir = argv[2];
  std::vector<int> lat = getiv(kv, "lattice"), bc = getiv(kv, "bc");
  if (lat.size() != 4) { fprintf(stderr, "lattice missing\n"); return 2; }
  if (bc.size() != 4) bc = std::vector<int>{1, 1, 1, -1};
  const int Ls = geti(kv, "Ls", 16);
  const int nthreads = geti(kv, "threads", 1);

  int one = 1;
  char** fake_argv = argv;
  bridge_initialize(&one, &fake_argv);
  bridge_setup(lat, std::vector<int>(4, 1), nthreads, 3, "stdout", "Crucial");
  if (!init_alt_QXS()) {
    fprintf(stderr, "init_alt_QXS failed\n");
    return 3;
  }
  const int Nvol = CommonParameters::Nvol(), Nvol2 = Nvol / 2;
  Field_G U(Nvol, 4);
  Field b(24, Nvol2, Ls);
  if (!read_bin(in_dir + "/gauge.bin", U.ptr(0), size_t(18) * Nvol * 4) ||
      !read_bin(in_dir + "/src.bin", b.ptr(0), size_t(24) * Nvol2 * Ls)) {
    fprintf(stderr, "input files missing or short\n");
    return 2;
  }

  Parameters params_fopr;
  params_fopr.set_string("fermion_type", "Domainwall_5din_eo");
  params_fopr.set_string("gamma_matrix_type", "Dirac");
  params_fopr.set_double("quark_mass", getd(kv, "mq", 0.01));
  params_fopr.set_double("domain_wall_height", getd(kv, "M0", 1.8));
  params_fopr.set_int("extent_of_5th_dimension", Ls);
  params_fopr.set_int_vector("boundary_condition", bc);
  params_fopr.set_double("coefficient_b", getd(kv, "b", 1.0));
  params_fopr.set_double("coefficient_c", getd(kv, "c", 0.0));
  params_fopr.set_string("verbose_level", "Crucial");

  // The solver's own rates come from its two operators' DdagD (the FP64
  // outer residual and the FP32 inner CG step); one bounded solve (one outer
  // iteration of one inner iteration: maximum_number_of_iteration = 1 with
  // one restart, which Fprop_alt_Standard_eo_Richardson::init hands to the
  // inner CG and ASolver_Richardson takes as its own bound) shows the
  // whole solver running on these inputs and what one outer step costs.
  AFopr<AFIELD_d>* fd = AFopr<AFIELD_d>::New("Domainwall_5din_eo", params_fopr);
  AFopr<AFIELD_f>* ff = AFopr<AFIELD_f>::New("Domainwall_5din_eo", params_fopr);
  if (!fd || !ff) {
    fprintf(stderr, "factory has no Domainwall_5din_eo for AField<REAL,QXS>\n");
    return 3;
  }
  fd->set_config(&U);
  ff->set_config(&U);
  const int nin = fd->field_nin(), nvol = fd->field_nvol(), nex = fd->field_nex();
  AFIELD_d bq(nin, nvol, nex), xq(nin, nvol, nex);
  fd->convert(bq, b);

  const int reps = geti(kv, "reps", 1);
  const double t_d = time_ddagd<AFIELD_d>(fd, reps);
  const double t_f = time_ddagd<AFIELD_f>(ff, reps);

  Parameters ps;
  ps.set_string("solver_type", "CG");
  ps.set_int("maximum_number_of_iteration", 1);
  ps.set_int("maximum_number_of_restart", 1);
  ps.set_double("convergence_criterion_squared", 1.0e-20);
  ps.set_string("use_initial_guess", "false");
  ps.set_string("verbose_level", "Crucial");
  Fprop_alt_Standard_eo_Richardson<AFIELD_d, AFIELD_f> fprop(params_fopr, ps);
  fprop.set_config(&U);
  int nconv = -1;
  double diff = -1.0;
  const double t0 = now();
  fprop.invert_DdagD_even(xq, bq, nconv, diff);
  const double t1 = now() - t0;
  printf("ddagd_f64_seconds %.6e\n", t_d);
  printf("ddagd_f32_seconds %.6e\n", t_f);
  printf("solve_1x1_seconds %.6e\n", t1);
  printf("threads %d\n", nthreads);
  delete fd;
  delete ff;
  return 0;
}
