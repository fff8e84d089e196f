// exasim_b200_<model>: the solver as an executable, in place of the reference's
// cput2cEXASIM / gput2cEXASIM for an HDG problem (backend/Main/main.cpp, Main/exasim.hpp).
//
//   exasim_b200_<model> <datain dir> <output prefix> [device]
//
// reads <datain dir>/{app,master,mesh,sol}.bin as text2code writes them, solves through the
// library's C ABI (steady: Newton; time dependent: every DIRK step of app.bin), and writes
// <output prefix>udg_np0.bin and <output prefix>uhat_np0.bin in the reference's format
// (backend/Solution/solution.h:45-58, 109-117; solution.cpp:726-752): a header of three
// float64 words (npe, nc, ne) or (ncu, npf, nf), then one snapshot of udg (all nc fields, or
// u alone with saveSolOpt 0) and of uhat per saved step.  Steady problems save once; time-
// dependent ones after every saveSolFreq-th step.  With the reference's default prefix
// "dataout/out" the files are dataout/outudg_np0.bin and dataout/outuhat_np0.bin.
// Exit status 0, or 1 with the library's message on stderr.
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <string>
#include <vector>

#include "../../include/exasim_b200.h"

namespace {

std::vector<double> read_words(const std::string& fn) {
  std::ifstream f(fn, std::ios::binary | std::ios::ate);
  if (!f) {
    std::fprintf(stderr, "cannot open %s\n", fn.c_str());
    std::exit(1);
  }
  std::vector<double> w((size_t)f.tellg() / sizeof(double));
  f.seekg(0);
  f.read(reinterpret_cast<char*>(w.data()), (std::streamsize)(w.size() * sizeof(double)));
  return w;
}

// part p of an Exasim blob [lsize, nsize(lsize), parts...]; empty if absent
std::vector<double> part(const std::vector<double>& b, int p) {
  if (b.empty()) return {};
  const long long ls = (long long)b[0];
  if (p >= ls || 1 + ls > (long long)b.size()) return {};
  long long o = 1 + ls;
  for (int i = 0; i < p; ++i) o += (long long)b[1 + i];
  const long long n = (long long)b[1 + p];
  if (o + n > (long long)b.size()) return {};
  return std::vector<double>(b.begin() + o, b.begin() + o + n);
}

void check(int st, const char* what) {
  if (st != 0) {
    std::fprintf(stderr, "%s: %s\n", what, exa_last_error());
    std::exit(1);
  }
}

struct Output {
  std::ofstream f;
  void open(const std::string& fn, double a0, double a1, double a2) {
    f.open(fn, std::ios::binary);
    if (!f) {
      std::fprintf(stderr, "cannot write %s\n", fn.c_str());
      std::exit(1);
    }
    const double h[3] = {a0, a1, a2};
    f.write(reinterpret_cast<const char*>(h), sizeof(h));
  }
  void write(const std::vector<double>& v) { f.write(reinterpret_cast<const char*>(v.data()), (std::streamsize)(v.size() * sizeof(double))); }
};

}  // namespace

int main(int argc, char** argv) {
  if (argc < 3) {
    std::fprintf(stderr, "usage: %s <datain dir> <output prefix> [device]\n", argv[0]);
    return 1;
  }
  const std::string din = std::string(argv[1]) + "/", prefix = argv[2];
  const int device = argc > 3 ? std::atoi(argv[3]) : 0;
  const std::vector<double> app = read_words(din + "app.bin"), master = read_words(din + "master.bin"),
                            mesh = read_words(din + "mesh.bin"), sol = read_words(din + "sol.bin");
  exa_ctx* ctx = nullptr;
  check(exa_create(app.data(), (long long)app.size(), master.data(), (long long)master.size(), mesh.data(),
                   (long long)mesh.size(), sol.data(), (long long)sol.size(), device, &ctx),
        "exa_create");
  long long sz[16];
  check(exa_sizes(ctx, sz), "exa_sizes");
  const long long ne = sz[0], nf = sz[1], npe = sz[3], npf = sz[4], nc = sz[6], ncu = sz[7], nuh = sz[11];
  // app.bin: flag part 1 (tdep first), problem part 2 (nstage 4, saveSolFreq 17, saveSolOpt 18), dt part 4
  const std::vector<double> flag = part(app, 1), prob = part(app, 2), dt = part(app, 4);
  const bool tdep = (!flag.empty() && flag[0] != 0.0) || (!dt.empty() && dt[0] > 0.0);
  const int nstage = prob.size() > 4 ? (int)prob[4] : 1;
  const int freq = prob.size() > 17 && prob[17] > 0 ? (int)prob[17] : 1;
  const int opt = prob.size() > 18 ? (int)prob[18] : 1;
  const long long ncs = opt == 0 ? ncu : nc;  // fields saved per node

  Output oudg, ouh;
  oudg.open(prefix + "udg_np0.bin", (double)npe, (double)ncs, (double)ne);
  ouh.open(prefix + "uhat_np0.bin", (double)ncu, (double)npf, (double)nf);
  std::vector<double> udg((size_t)(npe * nc * ne)), uh((size_t)nuh);
  auto save = [&]() {
    check(exa_get_field(ctx, "udg", udg.data(), (long long)udg.size()), "exa_get_field udg");
    check(exa_get_field(ctx, "uh", uh.data(), (long long)uh.size()), "exa_get_field uh");
    if (ncs == nc) {
      oudg.write(udg);
    } else {
      std::vector<double> u((size_t)(npe * ncu * ne));
      for (long long e = 0; e < ne; ++e)
        for (long long k = 0; k < ncu; ++k)
          for (long long i = 0; i < npe; ++i) u[i + npe * (k + ncu * e)] = udg[i + npe * (k + nc * e)];
      oudg.write(u);
    }
    ouh.write(uh);
  };
  if (!tdep) {
    int its = 0;
    double nrm = 0.0;
    check(exa_newton(ctx, &its, &nrm), "exa_newton");
    std::printf("Newton: %d steps, residual norm %.6e\n", its, nrm);
    save();
  } else {
    for (int istep = 0; istep < (int)dt.size(); ++istep) {
      for (int j = 0; j < nstage; ++j) {
        int its = 0;
        double nrm = 0.0;
        check(exa_dirk_stage(ctx, istep, j, &its, &nrm), "exa_dirk_stage");
      }
      std::printf("step %d done\n", istep + 1);
      if ((istep + 1) % freq == 0) save();
    }
  }
  exa_destroy(ctx);
  return 0;
}
