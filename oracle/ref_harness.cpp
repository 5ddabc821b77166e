// Harness that drives the reference Bridge++ corelib CPU path (compiled from
// its own sources by oracle/Makefile.ref) so that its outputs can serve as
// golden vectors for the oracle and as the timed CPU baseline.
//
// This file is test infrastructure: nothing in the product links it.
//
// Usage:  ref_harness <command> <params.txt> <in_dir> <out_dir>
//
// params.txt holds "key value [value...]" lines:
//   lattice Nx Ny Nz Nt      Ls n      mq x      M0 x      b x     c x
//   alpha x                  bc bx by bz bt      threads n
//   tol x (squared)          maxiter n           sigma s0 s1 ...
//   reps n                   modes Deo Doe ...
// Inputs (raw little-endian float64):
//   in_dir/gauge.bin  lexical links, Field_G(Nvol, 4) layout
//                     re/im + 2*(col + 3*row) + 18*(site + Nvol*mu)
//   in_dir/src.bin    5D half-lattice spinor, Field(24, Nvol/2, Ls) layout
//                     re/im + 2*(color + 3*spin) + 24*(site + Nvol2*s)
// Commands:
//   modes   : applies AFopr_Domainwall_eo<Field>::mult / mult_dag for every
//             listed mode (reference src/lib/Fopr/afopr_Domainwall_eo-tmpl.h)
//             and writes out_dir/<mode>.bin ("dag_<mode>" for mult_dag).
//   cg      : Solver_CG on mode DdagD (src/lib/Solver/solver_CG.cpp), writes
//             out_dir/cg_x.bin and out_dir/cg_info.txt.
//   shiftcg : Shiftsolver_CG on DdagD + sigma_i (src/lib/Solver/
//             shiftsolver_CG.cpp), writes out_dir/shift_<i>.bin.
//   time    : times `reps` applications of mode(s) inside an OpenMP parallel
//             region, prints "mode seconds_per_call".
//   force   : Force_F_Domainwall_eo (src/lib/Force/Fermion/
//             force_F_Domainwall_eo.cpp:150-327) with eta = src.bin and
//             zeta = in_dir/src2.bin: writes force_udiv1 in modes "H" and
//             "Hdag" (force_H.bin, force_Hdag.bin) and force_udiv(eta)
//             (force_udiv.bin), lexical Field_G(Nvol, 4) layout.
//   smear   : stout smearing Smear_APE + Projection_Stout_SU3 under
//             Director_Smear (rho, nsmear): writes smear_<i>.bin for the
//             levels i = 1..nsmear, and the Jacobian chain of ForceSmear_APE
//             (src/lib/Smear/forceSmear_APE.cpp, projection_Stout_SU3.cpp
//             force_recursive) applied to in_dir/sigma.bin from the top
//             level down to the thin links: jacobian.bin.
//   traj    : one 2+1-flavour HMC trajectory with the action set, smearing
//             and nested integrator of the reference's benchmark driver
//             (benchmark_hmc_dwf_corelib/hmc_dwf_eo.cpp:155-352): rational
//             ratio (PV / strange) and two Hasenbusch ratios (prec / light,
//             PV / prec), all on stout-smeared links, plus the rectangle
//             gauge action, under Builder_Integrator (Omelyan or Leapfrog)
//             and HMC_General::langevin / calc_Hamiltonian.  The Gaussian
//             fields the random-number generator hands out are recorded:
//             mom.bin (iP after the momentum heatbath), xi_<k>.bin (the
//             even-site noise of the k-th fermion action, Field(24, Nvol/2,
//             Ls)); the end links and momenta go to u_end.bin / mom_end.bin
//             and the Hamiltonians to traj.txt; force_<i>.bin holds each
//             action's force at the start links.  The rational coefficient
//             files (Math_Rational format) are read from in_dir.

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <sstream>
#include <fstream>
#include <vector>
#include <chrono>

#include "bridge_setup.h"
#include "Parameters/parameters.h"
#include "Parameters/commonParameters.h"
#include "ResourceManager/threadManager.h"
#include "Field/field.h"
#include "Field/field_G.h"
#include "Field/field_F.h"
#include "Fopr/fopr_Domainwall_eo.h"
#include "Solver/solver_CG.h"
#include "Solver/shiftsolver_CG.h"
#include "Force/Fermion/force_F_Domainwall_eo.h"
#include "Smear/projection_Stout_SU3.h"
#include "Smear/smear_APE.h"
#include "Smear/forceSmear_APE.h"
#include "Smear/director_Smear.h"
#include "Force/Gauge/force_G_Rectangle.h"
#include "Action/Gauge/action_G_Rectangle.h"
#include "IO/bridgeIO.h"
#include "Field/index_eo.h"
#include "Tools/randomNumbers_parallel.h"
#include "IO/gaugeConfig.h"
#include "Tools/randomNumbers_Mseries.h"
#include "Fopr/fopr_Smeared_eo.h"
#include "Force/Fermion/force_F_Smeared.h"
#include "Force/Fermion/force_F_Rational_Ratio.h"
#include "Action/Fermion/action_F_Ratio_eo.h"
#include "Action/Fermion/action_F_Rational_Ratio_eo.h"
#include "Measurements/Fermion/fprop_Standard_eo.h"
#include "HMC/action_list.h"
#include "HMC/builder_Integrator.h"
#include "HMC/hmc_General.h"
#include "Tools/randomNumbers_Mseries.h"
#include <unistd.h>

using Bridge::vout;

namespace {

typedef std::map<std::string, std::vector<std::string> > Kv;

Kv read_params(const char *path)
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

double getd(const Kv& kv, const char *k, double def)
{
  Kv::const_iterator it = kv.find(k);
  return (it == kv.end() || it->second.empty()) ? def : atof(it->second[0].c_str());
}

int geti(const Kv& kv, const char *k, int def)
{
  Kv::const_iterator it = kv.find(k);
  return (it == kv.end() || it->second.empty()) ? def : atoi(it->second[0].c_str());
}

std::vector<int> getiv(const Kv& kv, const char *k)
{
  std::vector<int> r;
  Kv::const_iterator it = kv.find(k);
  if (it != kv.end())
    for (size_t i = 0; i < it->second.size(); ++i) r.push_back(atoi(it->second[i].c_str()));
  return r;
}

void read_bin(const std::string& path, double *p, size_t n)
{
  FILE *f = fopen(path.c_str(), "rb");
  if (!f) { fprintf(stderr, "cannot open %s\n", path.c_str()); exit(2); }
  size_t got = fread(p, sizeof(double), n, f);
  fclose(f);
  if (got != n) { fprintf(stderr, "short read %s: %zu of %zu\n", path.c_str(), got, n); exit(2); }
}

void write_bin(const std::string& path, const double *p, size_t n)
{
  FILE *f = fopen(path.c_str(), "wb");
  if (!f) { fprintf(stderr, "cannot write %s\n", path.c_str()); exit(2); }
  fwrite(p, sizeof(double), n, f);
  fclose(f);
}

Parameters dwf_params(const Kv& kv)
{
  Parameters p;
  p.set_string("kernel_type", "Wilson");
  p.set_string("gamma_matrix_type", "Dirac");
  p.set_double("quark_mass", getd(kv, "mq", 0.01));
  p.set_double("domain_wall_height", getd(kv, "M0", 1.8));
  p.set_int("extent_of_5th_dimension", geti(kv, "Ls", 8));
  std::vector<int> bc = getiv(kv, "bc");
  if (bc.size() != 4) { bc.assign(4, 1); bc[3] = -1; }
  p.set_int_vector("boundary_condition", bc);
  p.set_double("coefficient_b", getd(kv, "b", 1.0));
  p.set_double("coefficient_c", getd(kv, "c", 0.0));
  p.set_double("parameter_alpha", getd(kv, "alpha", 1.0));
  p.set_string("verbose_level", "Crucial");
  return p;
}

// M-series generator that keeps a copy of every Gaussian field it hands out,
// so the same momenta and pseudofermion noise can drive another
// implementation of the trajectory.
class RecordingMseries : public RandomNumbers_Mseries {
 public:
  explicit RecordingMseries(int seed) : RandomNumbers_Mseries(seed) {}
  void gauss_lex_global(Field& f) {
    RandomNumbers::gauss_lex_global(f);
    record.push_back(f);
  }
  std::vector<Field> record;
};

Parameters rational_params(const Kv& kv, int np, int n_exp, int d_exp, double tol)
{
  Parameters p;
  p.set_int("number_of_poles", np);
  p.set_int("exponent_numerator", n_exp);
  p.set_int("exponent_denominator", d_exp);
  p.set_double("lower_bound", getd(kv, "rat_lo", 1e-2));
  p.set_double("upper_bound", getd(kv, "rat_hi", 3.16227766));
  p.set_int("maximum_number_of_iteration", geti(kv, "rat_maxiter", 10000));
  p.set_double("convergence_criterion_squared", tol);
  p.set_string("verbose_level", "Crucial");
  return p;
}

Parameters dwf_mass(const Kv& kv, const char *key)
{
  Parameters p = dwf_params(kv);
  p.set_double("quark_mass", getd(kv, key, 0.01));
  return p;
}

int run_traj(const Kv& kv, const std::string& in_dir, const std::string& out_dir, Field_G& Uorg)
{
  const int Nvol = CommonParameters::Nvol();
  const int Ls = geti(kv, "Ls", 8);
  const int np_md = geti(kv, "np_md", 16), np_h = geti(kv, "np_h", 24);
  const double tol_md = getd(kv, "tol_md", 1e-24), tol_h = getd(kv, "tol_h", 1e-24);
  const int cg_iter = geti(kv, "cg_maxiter", 100), cg_restart = geti(kv, "cg_restart", 100);

  // Math_Rational opens its coefficient files relative to the working directory
  std::string abs_out = out_dir;
  if (abs_out[0] != '/') {
    char cwd[4096];
    if (getcwd(cwd, sizeof(cwd))) abs_out = std::string(cwd) + "/" + out_dir;
  }
  if (chdir(in_dir.c_str()) != 0) { fprintf(stderr, "cannot chdir %s\n", in_dir.c_str()); return 2; }

  // through Parameters, as Action::New does in the driver: only this form
  // also configures the action's Force_G_Rectangle
  Parameters pg;
  pg.set_double("beta", getd(kv, "beta", 2.13));
  pg.set_double("c_plaq", getd(kv, "c_plaq", 3.648));
  pg.set_double("c_rect", getd(kv, "c_rect", -0.331));
  pg.set_string("verbose_level", "Crucial");
  Action_G_Rectangle action_G(pg);

  Projection_Stout_SU3 proj;
  Smear_APE smear(&proj);
  smear.set_parameters(getd(kv, "rho", 0.1));
  ForceSmear_APE force_smear(&proj);
  force_smear.set_parameters(getd(kv, "rho", 0.1));
  Director_Smear dr_smear(&smear);
  dr_smear.set_parameters(geti(kv, "nsmear", 2));

  // one flavour: rational ratio det[(B^dag B)^(1/2) / (A^dag A)^(1/2)],
  // B = strange domain wall, A = Pauli-Villars (mass mq_pv)
  Fopr_Domainwall_eo fopr_nf1(dwf_mass(kv, "mq_s"));
  Force_F_Domainwall_eo force_nf1(dwf_mass(kv, "mq_s"));
  Fopr_Domainwall_eo fopr_nf1_pv(dwf_mass(kv, "mq_pv"));
  Force_F_Domainwall_eo force_nf1_pv(dwf_mass(kv, "mq_pv"));
  Parameters prat_md;
  prat_md.set_Parameters("Fopr_Rational_numerator_MD", rational_params(kv, np_md, 1, 4, tol_md));
  prat_md.set_Parameters("Fopr_Rational_denominator_MD", rational_params(kv, np_md, -1, 2, tol_md));
  Force_F_Rational_Ratio force_rat(&fopr_nf1_pv, &force_nf1_pv, &fopr_nf1, &force_nf1, prat_md);
  Fopr_Smeared_eo fopr_nf1_smr(&fopr_nf1, &dr_smear);
  Fopr_Smeared_eo fopr_nf1_pv_smr(&fopr_nf1_pv, &dr_smear);
  Force_F_Smeared force_rat_smr(&force_rat, &force_smear, &dr_smear);
  Parameters prat_h;
  prat_h.set_Parameters("Fopr_Rational_numerator_calcH", rational_params(kv, np_h, 1, 4, tol_h));
  prat_h.set_Parameters("Fopr_Rational_denominator_calcH", rational_params(kv, np_h, -1, 2, tol_h));
  Action_F_Rational_Ratio_eo action_nf1(&fopr_nf1_pv_smr, &fopr_nf1_smr, &force_rat_smr, prat_h);

  // two flavours: Hasenbusch ratios prec/light and PV/prec
  Fopr_Domainwall_eo fopr_l(dwf_mass(kv, "mq_l"));
  Force_F_Domainwall_eo force_l(dwf_mass(kv, "mq_l"));
  Fopr_Domainwall_eo fopr_h(dwf_mass(kv, "mq_h"));
  Force_F_Domainwall_eo force_h(dwf_mass(kv, "mq_h"));
  Fopr_Domainwall_eo fopr_pv(dwf_mass(kv, "mq_pv"));
  Force_F_Domainwall_eo force_pv(dwf_mass(kv, "mq_pv"));
  Fopr_Smeared_eo fopr_l_smr(&fopr_l, &dr_smear);
  Fopr_Smeared_eo fopr_h_smr(&fopr_h, &dr_smear);
  Fopr_Smeared_eo fopr_pv_smr(&fopr_pv, &dr_smear);
  Force_F_Smeared force_l_smr(&force_l, &force_smear, &dr_smear);
  Force_F_Smeared force_h_smr(&force_h, &force_smear, &dr_smear);
  Force_F_Smeared force_pv_smr(&force_pv, &force_smear, &dr_smear);
  Solver_CG solver_l_md(&fopr_l_smr), solver_h_md(&fopr_h_smr);
  Solver_CG solver_l_h(&fopr_l_smr), solver_h_h(&fopr_h_smr), solver_pv_h(&fopr_pv_smr);
  solver_l_md.set_parameters(cg_iter, cg_restart, tol_md, false);
  solver_h_md.set_parameters(cg_iter, cg_restart, tol_md, false);
  solver_l_h.set_parameters(cg_iter, cg_restart, tol_h, false);
  solver_h_h.set_parameters(cg_iter, cg_restart, tol_h, false);
  solver_pv_h.set_parameters(cg_iter, cg_restart, tol_h, false);
  Fprop_Standard_eo fprop_l_md(&solver_l_md), fprop_h_md(&solver_h_md);
  Fprop_Standard_eo fprop_l_h(&solver_l_h), fprop_h_h(&solver_h_h), fprop_pv_h(&solver_pv_h);
  Action_F_Ratio_eo action_nf2(&fopr_h_smr, &force_h_smr, &fopr_l_smr, &force_l_smr,
                               &fprop_h_h, &fprop_l_md, &fprop_l_h);
  Action_F_Ratio_eo action_nf2_prec(&fopr_pv_smr, &force_pv_smr, &fopr_h_smr, &force_h_smr,
                                    &fprop_pv_h, &fprop_h_md, &fprop_h_h);

  std::vector<int> level = getiv(kv, "level");
  std::vector<int> nstep = getiv(kv, "nstep");
  if (level.size() != 4 || nstep.empty()) { fprintf(stderr, "level/nstep missing\n"); return 2; }
  ActionList actions(int(nstep.size()));
  actions.append(level[0], &action_nf1);
  actions.append(level[1], &action_nf2);
  actions.append(level[2], &action_nf2_prec);
  actions.append(level[3], &action_G);
  std::vector<Director *> directors(1, &dr_smear);

  Parameters pint;
  Kv::const_iterator iit = kv.find("integrator");
  pint.set_string("integrator", iit == kv.end() ? std::string("Omelyan") : iit->second[0]);
  pint.set_int("number_of_levels", int(nstep.size()));
  pint.set_int_vector("level_of_actions", level);
  pint.set_int_vector("number_of_steps", nstep);
  pint.set_int("order_of_exp_iP", geti(kv, "nprec", 8));
  pint.set_double("lambda_Omelyan", getd(kv, "lambda", 0.1931833275));
  pint.set_string("verbose_level", "Crucial");
  Builder_Integrator builder(actions, directors, pint);
  Integrator *integrator = builder.build();

  RecordingMseries rand(geti(kv, "seed", 1234567));
  Parameters phmc;
  phmc.set_double("trajectory_length", getd(kv, "tau", 1.0));
  phmc.set_string("Metropolis_test", "false");
  phmc.set_string("verbose_level", "Crucial");
  HMC_General hmc(actions, directors, integrator, &rand, phmc);

  // HMC_General::update (src/lib/HMC/hmc_General.cpp) without the Metropolis
  // step, with the random fields and both Hamiltonians kept
  Field_G U(Uorg);
  ActionSet all = actions.get_actions();
  for (size_t i = 0; i < all.size(); ++i) all[i]->set_config(&U);
  Field_G iP(Nvol, 4);
  const double H0 = hmc.langevin(iP, U);
  const size_t ng = size_t(18) * Nvol * 4;
  write_bin(abs_out + "/mom.bin", iP.ptr(0), ng);
  Index_eo index;
  int k = 0;
  for (size_t r = 0; r < rand.record.size(); ++r) {
    if (rand.record[r].nin() != 24) continue;     // the momentum draw (8 reals per link)
    Field xi(24, Nvol / 2, Ls);
    index.convertField(xi, rand.record[r], 0);
    char name[64];
    snprintf(name, sizeof(name), "/xi_%d.bin", k++);
    write_bin(abs_out + name, xi.ptr(0), size_t(24) * (Nvol / 2) * Ls);
  }
  std::vector<double> h_start(all.size());
  for (size_t i = 0; i < all.size(); ++i) h_start[i] = all[i]->calcH();
  // each action's force (Action::force, after mult_generator) at the start
  for (size_t i = 0; i < all.size(); ++i) {
    Field_G F(Nvol, 4);
    all[i]->force(F);
    char name[64];
    snprintf(name, sizeof(name), "/force_%zu.bin", i);
    write_bin(abs_out + name, F.ptr(0), ng);
  }
  integrator->evolve(getd(kv, "tau", 1.0), iP, U);
  const double H1 = hmc.calc_Hamiltonian(iP, U);
  std::vector<double> h_end(all.size());
  for (size_t i = 0; i < all.size(); ++i) h_end[i] = all[i]->calcH();
  write_bin(abs_out + "/u_end.bin", U.ptr(0), ng);
  write_bin(abs_out + "/mom_end.bin", iP.ptr(0), ng);
  FILE *f = fopen((abs_out + "/traj.txt").c_str(), "w");
  fprintf(f, "H0 %.17e\nH1 %.17e\ndH %.17e\n", H0, H1, H1 - H0);
  fprintf(f, "h_start");
  for (size_t i = 0; i < all.size(); ++i) fprintf(f, " %.17e", h_start[i]);
  fprintf(f, "\nh_end");
  for (size_t i = 0; i < all.size(); ++i) fprintf(f, " %.17e", h_end[i]);
  fprintf(f, "\n");
  fclose(f);
  return 0;
}

}  // namespace

// The benchmark driver's generator (random_number_type Mseries_parallel:
// RandomNumbers_parallel<RandomNumbers_Mseries>, one M-series stream per
// (z, t) plane): a fixed sequence of draws in the corelib Field layout, so a
// restatement of the generator can be checked stream against stream.
//   u.bin  uniform Field(2, Nvol, 1)          h.bin  gauss Field(8, Nvol, 4)
//   x.bin  gauss Field(24, Nvol, Ls)          h2.bin gauss Field(8, Nvol, 4)
//   after reset(seed + 1)
int run_rng(const Kv& kv, const std::string& out_dir)
{
  const int Nvol = CommonParameters::Nvol();
  const int Ls = geti(kv, "Ls", 8);
  const unsigned long seed = (unsigned long)geti(kv, "seed", 1234567);
  RandomNumbers_parallel<RandomNumbers_Mseries> rnd(seed);
  Field u(2, Nvol, 1), h(8, Nvol, 4), x(24, Nvol, Ls), h2(8, Nvol, 4);
  rnd.uniform_lex_global(u);
  rnd.gauss_lex_global(h);
  rnd.gauss_lex_global(x);
  rnd.reset(seed + 1);
  rnd.gauss_lex_global(h2);
  write_bin(out_dir + "/u.bin", u.ptr(0), size_t(2) * Nvol);
  write_bin(out_dir + "/h.bin", h.ptr(0), size_t(8) * Nvol * 4);
  write_bin(out_dir + "/x.bin", x.ptr(0), size_t(24) * Nvol * Ls);
  write_bin(out_dir + "/h2.bin", h2.ptr(0), size_t(8) * Nvol * 4);
  return 0;
}

// Gauge-configuration files through the reference's own readers/writers:
// in_dir/conf.txt (Text_4x4x4x8) is read onto the run's lattice and dumped
// (text_read.bin, native doubles), written as Binary (conf.bin) and read
// back (bin_read.bin).
int run_io(const std::string& in_dir, const std::string& out_dir)
{
  const int Nvol = CommonParameters::Nvol();
  const size_t ng = size_t(18) * Nvol * 4;
  Field_G U(Nvol, 4), V(Nvol, 4);
  GaugeConfig("Text_4x4x4x8").read(U, in_dir + "/conf.txt");
  write_bin(out_dir + "/text_read.bin", U.ptr(0), ng);
  GaugeConfig("Binary").write_file(U, out_dir + "/conf.bin");
  GaugeConfig("Binary").read(V, out_dir + "/conf.bin");
  write_bin(out_dir + "/bin_read.bin", V.ptr(0), ng);
  return 0;
}

int main(int argc, char **argv)
{
  if (argc < 5) {
    fprintf(stderr, "usage: %s <modes|cg|shiftcg|time|force|smear|gauge|traj|rng|io> params.txt in_dir out_dir\n", argv[0]);
    return 2;
  }
  const std::string cmd = argv[1];
  Kv kv = read_params(argv[2]);
  const std::string in_dir = argv[3], out_dir = argv[4];

  std::vector<int> lat = getiv(kv, "lattice");
  if (lat.size() != 4) { fprintf(stderr, "lattice missing\n"); return 2; }
  std::vector<int> grid(4, 1);
  const int nthreads = geti(kv, "threads", 1);

  int one = 1;
  char *fake_argv0 = argv[0];
  char **fake_argv = &fake_argv0;
  bridge_initialize(&one, &fake_argv);
  bridge_setup(lat, grid, nthreads, 3, "stdout", "Crucial");

  if (cmd == "rng") return run_rng(kv, out_dir);
  if (cmd == "io") return run_io(in_dir, out_dir);

  const int Nvol = CommonParameters::Nvol();
  const int Nvol2 = Nvol / 2;
  const int Ls = geti(kv, "Ls", 8);

  Field_G U(Nvol, 4);
  read_bin(in_dir + "/gauge.bin", U.ptr(0), size_t(18) * Nvol * 4);

  Parameters pf = dwf_params(kv);
  Fopr_Domainwall_eo fopr(pf);
  fopr.set_config(&U);

  if (cmd == "traj") return run_traj(kv, in_dir, out_dir, U);

  const size_t nsp = size_t(24) * Nvol2 * Ls;
  Field src(24, Nvol2, Ls), out(24, Nvol2, Ls);
  read_bin(in_dir + "/src.bin", src.ptr(0), nsp);

  Kv::const_iterator mit = kv.find("modes");
  std::vector<std::string> modes;
  if (mit != kv.end()) modes = mit->second;

  if (cmd == "modes") {
    for (size_t i = 0; i < modes.size(); ++i) {
      std::string m = modes[i];
      bool dag = false;
      if (m.compare(0, 4, "dag_") == 0) { dag = true; m = m.substr(4); }
      out.set(0.0);
      if (m == "Deo" || m == "Doe" || m == "Dee" || m == "Doo" ||
          m == "Dee_inv" || m == "Doo_inv") {
        if (dag) fopr.mult_dag(out, src, m); else fopr.mult(out, src, m);
      } else if (m == "gm5R") {
        fopr.mult_gm5R(out, src);
      } else if (m == "R") {
        fopr.mult_R(out, src);
      } else {
        fopr.set_mode(m);
        if (dag) fopr.mult_dag(out, src); else fopr.mult(out, src);
      }
      write_bin(out_dir + "/" + modes[i] + ".bin", out.ptr(0), nsp);
    }
  } else if (cmd == "cg") {
    fopr.set_mode("DdagD");
    Solver_CG solver(&fopr);
    solver.set_parameters(geti(kv, "maxiter", 10000), 1, getd(kv, "tol", 1e-20), false);
    int nconv = 0;
    double diff = 0.0;
    solver.solve(out, src, nconv, diff);
    write_bin(out_dir + "/cg_x.bin", out.ptr(0), nsp);
    FILE *f = fopen((out_dir + "/cg_info.txt").c_str(), "w");
    fprintf(f, "nconv %d\ndiff %.17e\n", nconv, diff);
    fclose(f);
  } else if (cmd == "shiftcg") {
    fopr.set_mode("DdagD");
    Kv::const_iterator sit = kv.find("sigma");
    std::vector<double> sigma;
    for (size_t i = 0; i < sit->second.size(); ++i) sigma.push_back(atof(sit->second[i].c_str()));
    Shiftsolver_CG solver(&fopr, geti(kv, "maxiter", 10000), getd(kv, "tol", 1e-20));
    std::vector<Field> xs(sigma.size(), Field(24, Nvol2, Ls));
    int nconv = 0;
    double diff = 0.0;
    solver.solve(xs, sigma, src, nconv, diff);
    for (size_t i = 0; i < sigma.size(); ++i) {
      char name[64];
      snprintf(name, sizeof(name), "/shift_%zu.bin", i);
      write_bin(out_dir + name, xs[i].ptr(0), nsp);
    }
    FILE *f = fopen((out_dir + "/shift_info.txt").c_str(), "w");
    fprintf(f, "nconv %d\ndiff %.17e\n", nconv, diff);
    fclose(f);
  } else if (cmd == "force") {
    Field src2(24, Nvol2, Ls);
    read_bin(in_dir + "/src2.bin", src2.ptr(0), nsp);
    Force_F_Domainwall_eo force(pf);
    force.set_config(&U);
    Field_G F(Nvol, 4);
    const size_t nf = size_t(18) * Nvol * 4;
    force.set_mode("H");
    force.force_udiv1(F, src2, src);
    write_bin(out_dir + "/force_H.bin", F.ptr(0), nf);
    force.set_mode("Hdag");
    force.force_udiv1(F, src, src2);
    write_bin(out_dir + "/force_Hdag.bin", F.ptr(0), nf);
    force.force_udiv(F, src);
    write_bin(out_dir + "/force_udiv.bin", F.ptr(0), nf);
  } else if (cmd == "gauge") {
    // Force_G_Rectangle::force_core, Action_G_Rectangle::calcH and the link
    // update W = exp(alpha iP) U of Integrator_UpdateU (mult_exp_Field_G)
    const double beta = getd(kv, "beta", 2.13);
    const double c_plaq = getd(kv, "c_plaq", 3.648);
    const double c_rect = getd(kv, "c_rect", -0.331);
    const double alpha = getd(kv, "alpha", 0.1);
    const int nprec = geti(kv, "nprec", 8);
    const size_t ng = size_t(18) * Nvol * 4;
    Force_G_Rectangle fg;
    fg.set_parameters(beta, c_plaq, c_rect);
    fg.set_config(&U);
    Field_G F(Nvol, 4);
    F.set(0.0);
    fg.force_core(F);
    write_bin(out_dir + "/gforce.bin", F.ptr(0), ng);
    Action_G_Rectangle act;
    act.set_parameters(beta, c_plaq, c_rect);
    act.set_config(&U);
    const double H = act.calcH();
    FILE *f = fopen((out_dir + "/gauge_H.txt").c_str(), "w");
    fprintf(f, "%.17e\n", H);
    fclose(f);
    Field_G iP(Nvol, 4);
    read_bin(in_dir + "/mom.bin", iP.ptr(0), ng);
    Field_G W(Nvol, 4);
    mult_exp_Field_G(W, alpha, iP, U, nprec);
    write_bin(out_dir + "/update.bin", W.ptr(0), ng);
  } else if (cmd == "smear") {
    const double rho = getd(kv, "rho", 0.1);
    const int nsmear = geti(kv, "nsmear", 2);
    Projection_Stout_SU3 proj;
    Smear_APE smear(&proj);
    smear.set_parameters(rho);
    Director_Smear dr(&smear);
    dr.set_parameters(nsmear);
    dr.set_config(&U);
    const size_t ng = size_t(18) * Nvol * 4;
    for (int i = 1; i <= nsmear; ++i) {
      char name[64];
      snprintf(name, sizeof(name), "/smear_%d.bin", i);
      write_bin(out_dir + name, dr.get_config(i)->ptr(0), ng);
    }
    ForceSmear_APE fsmear(&proj);
    fsmear.set_parameters(rho);
    Field_G sigma(Nvol, 4), sigma_p(Nvol, 4);
    read_bin(in_dir + "/sigma.bin", sigma_p.ptr(0), ng);
    for (int i = nsmear - 1; i >= 0; --i) {
      fsmear.force_udiv(sigma, sigma_p, *dr.get_config(i));
      if (i > 0) copy(sigma_p, sigma);
    }
    write_bin(out_dir + "/jacobian.bin", sigma.ptr(0), ng);
  } else if (cmd == "time") {
    // "Deo"/"Doe"/... use mult(v, w, mode); "dag_<mode>" uses mult_dag;
    // composite modes (D, DdagD, ...) use set_mode + mult.
    const int reps = geti(kv, "reps", 10);
    const int warm = geti(kv, "warmup", 1);
    for (size_t i = 0; i < modes.size(); ++i) {
      std::string m = modes[i];
      bool dag = false;
      if (m.compare(0, 4, "dag_") == 0) { dag = true; m = m.substr(4); }
      const bool explicit_mode = (m == "Deo" || m == "Doe" || m == "Dee" || m == "Doo" ||
                                  m == "Dee_inv" || m == "Doo_inv");
      if (!explicit_mode) fopr.set_mode(m);
      // r < 0: `warm` untimed calls that touch all memory first
      std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
      for (int r = -warm; r < reps; ++r) {
        if (r == 0) t0 = std::chrono::steady_clock::now();
#pragma omp parallel
        {
          if (explicit_mode) {
            if (dag) fopr.mult_dag(out, src, m); else fopr.mult(out, src, m);
          } else {
            if (dag) fopr.mult_dag(out, src); else fopr.mult(out, src);
          }
        }
      }
      std::chrono::steady_clock::time_point t1 = std::chrono::steady_clock::now();
      double sec = std::chrono::duration<double>(t1 - t0).count() / reps;
      printf("%s %.9e\n", modes[i].c_str(), sec);
    }
  } else {
    fprintf(stderr, "unknown command %s\n", cmd.c_str());
    return 2;
  }
  fflush(stdout);
  return 0;
}
