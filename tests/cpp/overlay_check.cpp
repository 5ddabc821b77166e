// Check driver of the reference-side overlay (lqcd-dwf-hmc_b200/overlay):
// the reference's own templates run on the B200 field and operator built
// through the reference's factory.
//
//   overlay_check <params.txt> <in_dir> <out_dir>
//
// params.txt: "key value..." lines: lattice, Ls, mq, M0, b, c, bc, threads,
// tol, maxiter, sigma (shifts), cmd (modes | cg | shiftcg | fprop),
// modes (for cmd modes).  in_dir holds gauge.bin (Field_G, Nvol x 4 x 18
// reals, lexical) and src.bin (the even-site source, Field(24, Nvol/2, Ls) in
// the reference's layout).  Outputs in the same layout: <mode>.bin,
// cg_x.bin, shift_<i>.bin, fprop_x.bin, and info.txt (iterations, diff).
//
//   modes   AFopr<AField<double,B200>>::New("Domainwall_5din_eo")->mult / mult_dag
//   cg      ASolver<AField<double,B200>>::New("CG", fopr) on DdagD
//           (src/lib_alt/Solver/asolver_CG-tmpl.h)
//   shiftcg AShiftsolver_CG<AField<double,B200>, AFopr<...>> on DdagD + sigma
//           (src/lib/Solver/ashiftsolver_CG-tmpl.h)
//   fprop   Fprop_alt_Standard_eo_Richardson<AField<double,B200>, AField<float,B200>>
//           ::invert_DdagD_even (FP64 Richardson, FP32 inner CG;
//           src/lib_alt/Measurements/Fermion/fprop_alt_Standard_eo_Richardson-tmpl.h)
#define DIRECTOR_ALT_SMEARED_IMPLEMENTED
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "bridge_setup.h"
#include "lib/Field/field.h"
#include "lib/Field/field_G.h"
#include "lib/Parameters/commonParameters.h"
#include "lib/Parameters/parameters.h"
#include "lib/ResourceManager/threadManager.h"
#include "lib/Solver/ashiftsolver_CG.h"
#include "lib_alt/Smear/director_alt_Smear.h"
#include "lib_alt/Measurements/Fermion/fprop_alt_Standard_eo_Richardson.h"
#include "lib_alt/Solver/asolver.h"
#include "lib_alt_B200/Field/afield.h"
#include "lib_alt_B200/Fopr/afopr_Domainwall_5din_eo.h"
#include "lib_alt_B200/init_alt_B200.h"

typedef AField<double, B200> AFIELD_d;
typedef AField<float, B200> AFIELD_f;

static std::map<std::string, std::vector<std::string> > read_params(const std::string& path)
{
  std::map<std::string, std::vector<std::string> > kv;
  std::ifstream f(path.c_str());
  std::string line;
  while (std::getline(f, line)) {
    std::istringstream is(line);
    std::string key, v;
    if (!(is >> key)) continue;
    while (is >> v) kv[key].push_back(v);
  }
  return kv;
}

static void read_bin(const std::string& path, double *p, size_t n)
{
  FILE *f = fopen(path.c_str(), "rb");
  if (!f || fread(p, sizeof(double), n, f) != n) {
    fprintf(stderr, "cannot read %zu doubles from %s\n", n, path.c_str());
    exit(2);
  }
  fclose(f);
}

static void write_bin(const std::string& path, const double *p, size_t n)
{
  FILE *f = fopen(path.c_str(), "wb");
  if (!f || fwrite(p, sizeof(double), n, f) != n) {
    fprintf(stderr, "cannot write %s\n", path.c_str());
    exit(2);
  }
  fclose(f);
}

int main(int argc, char **argv)
{
  if (argc != 4) {
    fprintf(stderr, "usage: %s params.txt in_dir out_dir\n", argv[0]);
    return 2;
  }
  std::map<std::string, std::vector<std::string> > kv = read_params(argv[1]);
  const std::string in_dir = argv[2], out_dir = argv[3];
  std::vector<int> lat, bc;
  for (size_t i = 0; i < kv["lattice"].size(); ++i) lat.push_back(atoi(kv["lattice"][i].c_str()));
  for (size_t i = 0; i < kv["bc"].size(); ++i) bc.push_back(atoi(kv["bc"][i].c_str()));
  const int Ls = atoi(kv["Ls"][0].c_str());
  const int nthreads = kv.count("threads") ? atoi(kv["threads"][0].c_str()) : 1;
  const std::string cmd = kv["cmd"][0];

  int one = 1;
  char **fake_argv = argv;
  bridge_initialize(&one, &fake_argv);
  bridge_setup(lat, std::vector<int>(4, 1), nthreads, 3, "stdout", "Crucial");
  if (!init_alt_B200(0, 0)) {
    fprintf(stderr, "init_alt_B200 failed\n");
    return 3;
  }

  const int Nvol = CommonParameters::Nvol(), Nvol2 = Nvol / 2;
  Field_G U(Nvol, 4);
  read_bin(in_dir + "/gauge.bin", U.ptr(0), size_t(18) * Nvol * 4);
  Field b(24, Nvol2, Ls);
  read_bin(in_dir + "/src.bin", b.ptr(0), size_t(24) * Nvol2 * Ls);

  Parameters params_fopr;
  params_fopr.set_string("fermion_type", "Domainwall_5din_eo");
  params_fopr.set_string("gamma_matrix_type", "Dirac");
  params_fopr.set_double("quark_mass", atof(kv["mq"][0].c_str()));
  params_fopr.set_double("domain_wall_height", atof(kv["M0"][0].c_str()));
  params_fopr.set_int("extent_of_5th_dimension", Ls);
  params_fopr.set_int_vector("boundary_condition", bc);
  params_fopr.set_double("coefficient_b", atof(kv["b"][0].c_str()));
  params_fopr.set_double("coefficient_c", atof(kv["c"][0].c_str()));
  params_fopr.set_string("verbose_level", "Crucial");

  AFopr<AFIELD_d> *fopr = AFopr<AFIELD_d>::New("Domainwall_5din_eo", params_fopr);
  if (!fopr) {
    fprintf(stderr, "factory has no Domainwall_5din_eo for AField<double,B200>\n");
    return 3;
  }
  fopr->set_config(&U);
  const int nin = fopr->field_nin(), nvol = fopr->field_nvol(), nex = fopr->field_nex();
  AFIELD_d bq(nin, nvol, nex), xq(nin, nvol, nex);
  fopr->convert(bq, b);
  Field out(24, Nvol2, Ls);
  FILE *info = fopen((out_dir + "/info.txt").c_str(), "w");

  const double tol = kv.count("tol") ? atof(kv["tol"][0].c_str()) : 1e-24;
  const int maxiter = kv.count("maxiter") ? atoi(kv["maxiter"][0].c_str()) : 10000;

  if (cmd == "modes") {
    for (size_t i = 0; i < kv["modes"].size(); ++i) {
      std::string m = kv["modes"][i];
      const bool dag = m.compare(0, 4, "dag_") == 0;
      if (dag) m = m.substr(4);
      if (dag) fopr->mult_dag(xq, bq, m); else fopr->mult(xq, bq, m);
      fopr->reverse(out, xq);
      write_bin(out_dir + "/" + kv["modes"][i] + ".bin", out.ptr(0), out.size());
    }
  } else if (cmd == "cg") {
    Parameters ps;
    ps.set_string("solver_type", "CG");
    ps.set_int("maximum_number_of_iteration", maxiter);
    ps.set_int("maximum_number_of_restart", 1);
    ps.set_double("convergence_criterion_squared", tol);
    ps.set_string("initial_guess_mode", "ZERO");
    ps.set_string("verbose_level", "Crucial");
    ASolver<AFIELD_d> *solver = ASolver<AFIELD_d>::New("CG", fopr);
    solver->set_parameters(ps);
    fopr->set_mode("DdagD");
    int nconv = -1;
    double diff = -1.0;
#pragma omp parallel
    {
      solver->solve(xq, bq, nconv, diff);
    }
    fopr->reverse(out, xq);
    write_bin(out_dir + "/cg_x.bin", out.ptr(0), out.size());
    fprintf(info, "nconv %d\ndiff %.17e\n", nconv, diff);
    delete solver;
  } else if (cmd == "shiftcg") {
    std::vector<double> sigma;
    for (size_t i = 0; i < kv["sigma"].size(); ++i) sigma.push_back(atof(kv["sigma"][i].c_str()));
    std::vector<AFIELD_d> xs(sigma.size());
    for (size_t i = 0; i < xs.size(); ++i) xs[i].reset(nin, nvol, nex);
    fopr->set_mode("DdagD");
    AShiftsolver_CG<AFIELD_d, AFopr<AFIELD_d> > solver(fopr, maxiter, tol);
    int nconv = -1;
    double diff = -1.0;
    solver.solve(xs, sigma, bq, nconv, diff);
    for (size_t i = 0; i < xs.size(); ++i) {
      fopr->reverse(out, xs[i]);
      std::ostringstream name;
      name << out_dir << "/shift_" << i << ".bin";
      write_bin(name.str(), out.ptr(0), out.size());
    }
    fprintf(info, "nconv %d\ndiff %.17e\n", nconv, diff);
  } else if (cmd == "fprop") {
    Parameters ps;
    ps.set_string("solver_type", "CG");
    ps.set_int("maximum_number_of_iteration", maxiter);
    ps.set_int("maximum_number_of_restart", 40);
    ps.set_double("convergence_criterion_squared", tol);
    ps.set_string("use_initial_guess", "false");
    ps.set_string("verbose_level", "Crucial");
    Fprop_alt_Standard_eo_Richardson<AFIELD_d, AFIELD_f> fprop(params_fopr, ps);
    fprop.set_config(&U);
    int nconv = -1;
    double diff = -1.0;
    fprop.invert_DdagD_even(xq, bq, nconv, diff);
    fopr->reverse(out, xq);
    write_bin(out_dir + "/fprop_x.bin", out.ptr(0), out.size());
    fprintf(info, "nconv %d\ndiff %.17e\n", nconv, diff);
  } else {
    fprintf(stderr, "unknown cmd %s\n", cmd.c_str());
    return 2;
  }
  fclose(info);
  delete fopr;
  bridge_finalize();
  return 0;
}
