// exasim_b200_<model>: the solver as an executable, in place of the reference's
// cput2cEXASIM / gput2cEXASIM for an HDG or LDG problem (backend/Main/main.cpp, Main/exasim.hpp).
//
//   exasim_b200_<model> <datain dir> <output prefix> [restart] [device] [--checkpoint] [--vtu]
//
// reads <datain dir>/{app,master,mesh,sol}.bin as text2code writes them, solves through the
// library's C ABI (steady: Newton; time dependent: every DIRK step of app.bin), and writes
// <output prefix>udg_np0.bin and <output prefix>uhat_np0.bin in the reference's format
// (backend/Solution/solution.h:45-58, 109-117; solution.cpp:726-752): a header of three
// float64 words (npe, nc, ne) or (ncu, npf, nf), then one snapshot of udg (all nc fields, or
// u alone with saveSolOpt 0) and of uhat per saved step.  Steady problems save once; time-
// dependent ones after every saveSolFreq-th step.  With the reference's default prefix
// "dataout/out" the files are dataout/outudg_np0.bin and dataout/outuhat_np0.bin.  An LDG
// problem (problem[0] = 0: pseudo-transient solves of the element states) writes udg only.
//
// Restart (time-dependent problems; exasim.hpp:338-348, 387-393, 413-420): restart R > 0, from
// the argument or app.bin's timestepOffset (problem[19]), starts the step loop at time R dt[0]
// from the state in <output prefix>udg_t<R>_np0.bin and <output prefix>_uhat_t<R>_np0.bin,
// raw float64 arrays as ReadSolutions reads them (solution.cpp:804-828): u alone (npe ncu ne
// words, inserted into udg) with saveSolOpt 0, else all of udg; then uhat.  --checkpoint
// writes those two files, numbered by step + R, at every saved step, so a later run can
// restart from any of them.
//
// --vtu writes each saved snapshot for visualization as well (exa_vtu.h): <output prefix>vis.vtu
// for a steady problem; <output prefix>vis_<step>.vtu per saved step and <output prefix>vis.pvd,
// the time series, for a time-dependent one (the reference's SaveParaview names,
// solution.cpp:861-880).
// Exit status 0, or 1 with the library's message on stderr.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <string>
#include <vector>

#include "../../include/exasim_b200.h"
#include "exa_vtu.h"

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
  void open_raw(const std::string& fn) {
    f.open(fn, std::ios::binary);
    if (!f) {
      std::fprintf(stderr, "cannot write %s\n", fn.c_str());
      std::exit(1);
    }
  }
  void write(const std::vector<double>& v) { f.write(reinterpret_cast<const char*>(v.data()), (std::streamsize)(v.size() * sizeof(double))); }
};

}  // namespace

int main(int argc, char** argv) {
  std::vector<std::string> pos;
  bool checkpoint = false, vtu = false;
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    if (a == "--checkpoint") checkpoint = true;
    else if (a == "--vtu") vtu = true;
    else pos.push_back(a);
  }
  if (pos.size() < 2) {
    std::fprintf(stderr, "usage: %s <datain dir> <output prefix> [restart] [device] [--checkpoint] [--vtu]\n", argv[0]);
    return 1;
  }
  const std::string din = pos[0] + "/", prefix = pos[1];
  char* end = nullptr;
  const long rarg = pos.size() > 2 ? std::strtol(pos[2].c_str(), &end, 10) : 0;
  if (pos.size() > 2 && (end == pos[2].c_str() || *end != '\0' || rarg < 0)) {
    std::fprintf(stderr, "invalid restart value: %s\n", pos[2].c_str());
    return 1;
  }
  const int device = pos.size() > 3 ? std::atoi(pos[3].c_str()) : 0;
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
  const int offset = prob.size() > 19 ? (int)prob[19] : 0;
  const int restart = offset > 0 ? offset : (int)rarg;  // the reference's precedence (exasim.hpp:387-388)
  // an LDG run (problem[0] = 0) has no trace field: it writes and reads udg only
  // (solution.cpp:735-760, 824-850 write uhat for HDG alone)
  const bool ldg = !prob.empty() && prob[0] == 0.0;
  std::vector<double> udg((size_t)(npe * nc * ne)), uh((size_t)nuh);
  if (restart > 0) {
    if (!tdep || dt.empty()) {
      std::fprintf(stderr, "restart %d: app.bin is not time dependent\n", restart);
      return 1;
    }
    const std::string fu = prefix + "udg_t" + std::to_string(restart) + "_np0.bin";
    const std::string fh = prefix + "_uhat_t" + std::to_string(restart) + "_np0.bin";
    const std::vector<double> ru = read_words(fu), rh = ldg ? std::vector<double>() : read_words(fh);
    const size_t nu = (size_t)(npe * ncs * ne);
    if (ru.size() < nu || (!ldg && rh.size() < (size_t)nuh)) {
      std::fprintf(stderr, "restart %d: %s holds %zu words (needs %zu), %s %zu (needs %lld)\n", restart, fu.c_str(),
                   ru.size(), nu, fh.c_str(), rh.size(), nuh);
      return 1;
    }
    check(exa_get_field(ctx, "udg", udg.data(), (long long)udg.size()), "exa_get_field udg");
    if (ncs == nc) {
      std::copy(ru.begin(), ru.begin() + (long long)nu, udg.begin());
    } else {
      for (long long e = 0; e < ne; ++e)
        for (long long k = 0; k < ncu; ++k)
          for (long long i = 0; i < npe; ++i) udg[i + npe * (k + nc * e)] = ru[i + npe * (k + ncu * e)];
    }
    check(exa_set_field(ctx, "udg", udg.data(), (long long)udg.size()), "exa_set_field udg");
    if (!ldg) check(exa_set_field(ctx, "uh", rh.data(), nuh), "exa_set_field uh");
    check(exa_set_step_time(ctx, restart * dt[0]), "exa_set_step_time");
    std::printf("restart at step %d, time %g\n", restart, restart * dt[0]);
  }

  Output oudg, ouh;
  oudg.open(prefix + "udg_np0.bin", (double)npe, (double)ncs, (double)ne);
  if (!ldg) ouh.open(prefix + "uhat_np0.bin", (double)ncu, (double)npf, (double)nf);
  // visualization: the master element's lattice and the nodes' coordinates
  const std::vector<double> mnd = part(master, 0), xpe = part(master, 9), xdg = part(sol, 1);
  const int vnd = mnd.size() > 5 ? (int)mnd[0] : 0, vet = mnd.size() > 5 ? (int)mnd[1] : 0;
  const int vp = mnd.size() > 5 ? (int)mnd[3] : 0;
  const int ncx = npe * ne > 0 ? (int)(xdg.size() / (size_t)(npe * ne)) : 0;
  std::vector<std::string> vis_files;
  std::vector<double> vis_times;
  double tnow = 0.0;  // the time of the state being saved (time-dependent runs)
  auto visualize = [&](int step) {
    const std::string name = tdep ? "vis_" + std::to_string(step) + ".vtu" : "vis.vtu";
    if (!exa_vtu::write(prefix + name, vnd, vet, vp, (int)npe, xpe.data(), ne, ncx, xdg.data(), (int)nc, udg.data())) {
      std::fprintf(stderr, "cannot write %s%s\n", prefix.c_str(), name.c_str());
      std::exit(1);
    }
    vis_files.push_back(name);
    vis_times.push_back(tnow);
  };
  auto save = [&](int step) {
    check(exa_get_field(ctx, "udg", udg.data(), (long long)udg.size()), "exa_get_field udg");
    check(exa_get_field(ctx, "uh", uh.data(), (long long)uh.size()), "exa_get_field uh");
    std::vector<double> u;
    if (ncs != nc) {
      u.resize((size_t)(npe * ncu * ne));
      for (long long e = 0; e < ne; ++e)
        for (long long k = 0; k < ncu; ++k)
          for (long long i = 0; i < npe; ++i) u[i + npe * (k + ncu * e)] = udg[i + npe * (k + nc * e)];
    }
    const std::vector<double>& us = ncs == nc ? udg : u;
    oudg.write(us);
    if (!ldg) ouh.write(uh);
    if (vtu) visualize(step);
    if (checkpoint && step > 0) {
      // the restart files of this step, raw (solution.cpp:804-828 reads them so)
      Output cu, ch;
      cu.open_raw(prefix + "udg_t" + std::to_string(step) + "_np0.bin");
      cu.write(us);
      if (!ldg) {
        ch.open_raw(prefix + "_uhat_t" + std::to_string(step) + "_np0.bin");
        ch.write(uh);
      }
    }
  };
  if (!tdep) {
    int its = 0;
    double nrm = 0.0;
    check(exa_newton(ctx, &its, &nrm), "exa_newton");
    std::printf("Newton: %d steps, residual norm %.6e\n", its, nrm);
    save(0);
  } else {
    // the start time: app.bin's factor[0] (time), or R dt[0] on a restart (exasim.hpp:390-393)
    const std::vector<double> factor = part(app, 5);
    tnow = restart > 0 ? restart * dt[0] : (factor.empty() ? 0.0 : factor[0]);
    for (int istep = 0; istep < (int)dt.size(); ++istep) {
      for (int j = 0; j < nstage; ++j) {
        int its = 0;
        double nrm = 0.0;
        check(exa_dirk_stage(ctx, istep, j, &its, &nrm), "exa_dirk_stage");
      }
      tnow += dt[istep];
      std::printf("step %d done\n", istep + 1 + restart);
      if ((istep + 1) % freq == 0) save(istep + 1 + restart);
    }
    if (vtu && !exa_vtu::write_pvd(prefix + "vis.pvd", vis_files, vis_times)) {
      std::fprintf(stderr, "cannot write %svis.pvd\n", prefix.c_str());
      return 1;
    }
  }
  exa_destroy(ctx);
  return 0;
}
