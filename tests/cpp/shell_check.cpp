// Drives the C++ shells of include/b200dwf.hpp the way the reference's
// templates drive AFopr / ASolver / AShiftsolver: reads links and a source in
// the reference host layouts, applies mult(v, w, "DdagD"), runs CG and the
// multishift CG, and writes the results for the Python test to check.
//   shell_check <dir>  (dir holds params.txt, gauge.bin, src.bin)
#include <cstdio>
#include <fstream>
#include <string>
#include <vector>

#include "b200dwf.hpp"

static std::vector<double> read_bin(const std::string& path, size_t n) {
  std::vector<double> v(n);
  std::ifstream f(path, std::ios::binary);
  f.read(reinterpret_cast<char*>(v.data()), n * sizeof(double));
  return v;
}

static void write_bin(const std::string& path, const std::vector<double>& v) {
  std::ofstream f(path, std::ios::binary);
  f.write(reinterpret_cast<const char*>(v.data()), v.size() * sizeof(double));
}

int main(int argc, char** argv) {
  if (argc < 2) return 2;
  const std::string dir = argv[1];
  int L[4], Ls;
  double mq, M0;
  FILE* pf = std::fopen((dir + "/params.txt").c_str(), "r");
  if (!pf || std::fscanf(pf, "%d %d %d %d %d %lf %lf", &L[0], &L[1], &L[2], &L[3], &Ls, &mq, &M0) != 7) return 3;
  std::fclose(pf);
  const size_t nvol = (size_t)L[0] * L[1] * L[2] * L[3];
  const size_t nfield = 24 * (nvol / 2) * Ls;

  b200::ok(b200_init(0, 0));
  b200::AFopr_Domainwall_B200 fopr(L, Ls, mq, M0);
  std::vector<double> u = read_bin(dir + "/gauge.bin", 18 * 4 * nvol);
  std::vector<double> src = read_bin(dir + "/src.bin", nfield);
  fopr.set_config(u.data());

  b200::AField_B200<double> w(fopr), v(fopr), x(fopr);
  fopr.convert(w, src.data());
  fopr.set_mode("DdagD");
  fopr.mult(v, w);
  std::vector<double> out(nfield);
  fopr.reverse(out.data(), v);
  write_bin(dir + "/ddagd.bin", out);

  b200::ASolver_CG_B200<double> cg(fopr, 10000, 1.0e-20);
  int nconv = 0;
  double diff = 0.0;
  cg.solve(x, w, nconv, diff);
  fopr.reverse(out.data(), x);
  write_bin(dir + "/cg.bin", out);

  std::vector<double> sigma = {0.05, 0.2, 1.0};
  b200::AField_B200<double> x0(fopr), x1(fopr), x2(fopr);
  std::vector<b200::AField_B200<double>*> xs = {&x0, &x1, &x2};
  b200::AShiftsolver_CG_B200 ms(fopr, 10000, 1.0e-20);
  int nms = 0;
  double dms = 0.0;
  ms.solve(xs, sigma, w, nms, dms);
  fopr.reverse(out.data(), x1);
  write_bin(dir + "/shift1.bin", out);
  std::printf("cg %d %.3e shift %d %.3e norm2 %.17e\n", nconv, diff, nms, dms, w.norm2());
  return 0;
}
