// dmrg2_gpu: command-line driver, argv/stdout-compatible with the reference's
// gpu-rocm/dmrg2-gpu/src/test_dmrg2_gpu.cpp (argv `L chi_max n_sweeps [flags]`,
// lines "Final energy:", "Total wall time:", "env_build_sec: ... timer_scope:",
// known-answer PASS/FAIL with exit code 1 on failure or error). It calls the
// engine only through the C ABI of include/dmrg2_b200.h.
//
// Added flags: --delta --ng --onsite {reference,shifted} --schedule c1,c2,...
// --cutoff --krylov --lanczos-tol --restarts --seed --init {random,neel,product}
// --tol --json FILE --verbose
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <map>
#include <sstream>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/dmrg2_b200.h"
#include "mpo_builders.h"

using namespace dmrg2cli;

namespace {

struct Args {
  int L = 8, chi = 32, sweeps = 30;
  std::string model = "heisenberg";
  bool quiet = false, verbose = false;
  int n_max = 1;
  double E_J = 1.0, E_C = 0.5, phi = M_PI / 4, n_g = 0.0;
  std::string onsite = "reference";
  double J_tfim = 1.0, h_field = 1.0;
  double J1 = 1.0, J2 = 0.5, J3 = 0.25;
  double J_leg = 1.0, J_rung = 1.0;
  double delta = 1.0;
  std::vector<int> schedule;
  double cutoff = 0.0, tol = 1e-10, lanczos_tol = 0.0;
  int krylov = 0, restarts = 0, precision = 0, single_site = 0;
  unsigned long long seed = 42;
  std::string init;
  std::string json;
  std::string cmdline;
};

std::string fmt(double v) {
  char b[64];
  std::snprintf(b, sizeof(b), "%.17g", v);
  return b;
}

int fail(dmrg2_handle* h, const char* what) {
  std::fprintf(stderr, "ERROR: %s: %s\n", what, dmrg2_last_error(h));
  if (h) dmrg2_destroy(h);
  return 1;
}

void write_json(const Args& a, const Mpo& m, double energy, double wall, double env_s,
                const std::vector<dmrg2_sweep_report>& rep) {
  FILE* f = std::fopen(a.json.c_str(), "w");
  if (!f) {
    std::fprintf(stderr, "cannot write %s\n", a.json.c_str());
    return;
  }
  double flops = 0, hs = 0, tmax = 0;
  std::ostringstream es, ts;
  for (size_t i = 0; i < rep.size(); ++i) {
    flops += rep[i].heff_flops;
    hs += rep[i].heff_s;
    tmax = std::max(tmax, rep[i].trunc_err_max);
    es << (i ? ", " : "") << fmt(rep[i].energy);
    ts << (i ? ", " : "") << fmt(rep[i].trunc_err_max);
  }
  char stamp[32];
  std::time_t t = std::time(nullptr);
  std::strftime(stamp, sizeof(stamp), "%Y%m%d_%H%M%S", std::gmtime(&t));
  std::fprintf(f,
               "{\n  \"implementation\": \"dmrg2-b200\",\n  \"architecture\": \"b200\",\n"
               "  \"benchmark\": \"cli\",\n  \"timestamp\": \"%s\",\n  \"results\": [\n    {\n"
               "      \"impl\": \"dmrg2-b200\", \"model\": \"%s\", \"L\": %d, \"chi\": %d, \"sweeps\": %d,\n"
               "      \"arch\": \"b200\", \"benchmark\": \"cli\", \"threads\": 1, \"np\": 1, \"success\": true,\n"
               "      \"time\": %s, \"time_median\": %s, \"time_min\": %s, \"times\": [%s],\n"
               "      \"energy\": %s, \"energies\": [%s], \"repeats\": 1, \"successful_reps\": 1,\n"
               "      \"cmd\": \"%s\", \"timer_scope\": \"sweep_only\", \"env_build_sec\": %s,\n"
               "      \"sweep_energies\": [%s], \"trunc_err\": [%s], \"sweeps_run\": %d,\n"
               "      \"sweeps_per_s\": %s, \"heff_tflops\": %s, \"precision_form\": \"%s\"%s\n"
               "    }\n  ]\n}\n",
               stamp, m.name.c_str(), a.L, a.chi, a.sweeps, fmt(wall).c_str(), fmt(wall).c_str(),
               fmt(wall).c_str(), fmt(wall).c_str(), fmt(energy).c_str(), fmt(energy).c_str(),
               a.cmdline.c_str(), fmt(env_s).c_str(), es.str().c_str(), ts.str().c_str(),
               (int)rep.size(), fmt(wall > 0 ? rep.size() / wall : 0.0).c_str(),
               fmt(hs > 0 ? flops / hs * 1e-12 : 0.0).c_str(), a.precision ? "split_bf16" : "fp64",
               m.name == "josephson" ? (", \"nmax\": " + std::to_string(a.n_max)).c_str() : "");
  std::fclose(f);
}

int solve(const Args& a, const Mpo& m, bool default_neel, double exact, double exact_tol,
          bool have_exact) {
  dmrg2_config cfg;
  std::memset(&cfg, 0, sizeof(cfg));
  cfg.L = m.L;
  cfg.d = m.d;
  int chi_cap = a.chi;
  for (int c : a.schedule) chi_cap = std::max(chi_cap, c);
  cfg.chi_max = chi_cap;
  cfg.dtype = m.cplx ? DMRG2_C128 : DMRG2_F64;
  cfg.tol = a.tol;
  cfg.krylov_max = a.krylov;
  cfg.lanczos_tol = a.lanczos_tol;
  cfg.max_restarts = a.restarts;
  cfg.cutoff = a.cutoff;
  cfg.seed = a.seed;
  cfg.precision = a.precision;
  cfg.single_site = a.single_site;
  dmrg2_handle* h = nullptr;
  if (dmrg2_create(&cfg, &h) != DMRG2_OK) return fail(nullptr, "create");
  std::vector<const void*> W(m.L);
  for (int i = 0; i < m.L; ++i) W[i] = m.W[i].data();
  if (dmrg2_set_mpo(h, W.data(), m.Dl.data(), m.Dr.data(), DMRG2_LAYOUT_ROWMAJOR) != DMRG2_OK)
    return fail(h, "set_mpo");
  int kind = default_neel ? DMRG2_INIT_NEEL : DMRG2_INIT_RANDOM;
  if (a.init == "random") kind = DMRG2_INIT_RANDOM;
  else if (a.init == "neel") kind = DMRG2_INIT_NEEL;
  else if (a.init == "product") kind = DMRG2_INIT_PRODUCT;
  if (dmrg2_init_mps(h, kind, a.seed) != DMRG2_OK) return fail(h, "init_mps");
  std::vector<int> sched = a.schedule;
  if (sched.empty()) sched.assign(a.sweeps, a.chi);
  while ((int)sched.size() < a.sweeps) sched.push_back(sched.back());
  sched.resize(a.sweeps);
  std::vector<dmrg2_sweep_report> rep(a.sweeps);
  int n_run = 0;
  auto t0 = std::chrono::steady_clock::now();
  if (dmrg2_run(h, sched.data(), a.sweeps, rep.data(), a.sweeps, &n_run) != DMRG2_OK)
    return fail(h, "run");
  double total = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  double env_s = 0.0, energy = 0.0;
  dmrg2_get_env_build_seconds(h, &env_s);
  dmrg2_get_energy(h, &energy);
  rep.resize(n_run);
  double wall = total - env_s;
  std::printf("  Environment build: %.3f s\n", env_s);
  if (a.verbose)
    for (auto& r : rep)
      std::printf("  sweep %d chi=%d E=%.14f trunc=%.3e bond=%d wall=%.3f s heff=%.3f s svd=%.3f s\n",
                  r.sweep, r.chi_max, r.energy, r.trunc_err_max, r.max_bond, r.wall_s, r.heff_s,
                  r.svd_s);
  std::printf("Final energy: %.12f\n", energy);
  std::printf("Total wall time: %.3f s\n", wall);
  std::printf("  env_build_sec: %.3f  timer_scope: sweep_only\n", env_s);
  if (!a.json.empty()) write_json(a, m, energy, wall, env_s, rep);
  dmrg2_destroy(h);
  int ret = 0;
  if (!a.quiet && have_exact) {
    double err = std::fabs(energy - exact);
    std::printf("Exact energy: %.12f\n", exact);
    std::printf("Absolute error: %.2e\n", err);
    if (err < exact_tol) std::printf("PASS\n");
    else { std::printf("FAIL\n"); ret = 1; }
  }
  return ret;
}

void banner(const Args& a, const char* title, const Mpo& m, const std::string& extra) {
  if (a.quiet) return;
  std::printf("======================================\n%s\n======================================\n", title);
  std::printf("  L=%d, d=%d, chi_max=%d, D_mpo=%d, sweeps=%d\n", a.L, m.d, a.chi,
              m.L > 2 ? m.Dl[1] : m.Dr[0], a.sweeps);
  if (!extra.empty()) std::printf("%s\n", extra.c_str());
  std::printf("======================================\n\n");
}

}  // namespace

int main(int argc, char** argv) {
  Args a;
  for (int i = 0; i < argc; ++i) a.cmdline += (i ? " " : "") + std::string(argv[i]);
  int pos = 0;
  for (int i = 1; i < argc; ++i) {
    std::string s = argv[i];
    auto next = [&](const char* f) -> const char* {
      if (i + 1 >= argc) { std::fprintf(stderr, "Missing value for %s\n", f); std::exit(1); }
      return argv[++i];
    };
    if (s == "--josephson") { a.model = "josephson"; continue; }
    if (s == "--tfim") { a.model = "tfim"; continue; }
    if (s == "--j1j2") { a.model = "j1j2"; continue; }
    if (s == "--j1j2j3") { a.model = "j1j2j3"; continue; }
    if (s == "--ladder") { a.model = "ladder"; continue; }
    if (s == "--quiet") { a.quiet = true; continue; }
    if (s == "--verbose") { a.verbose = true; continue; }
    if (s == "--hfield") { a.h_field = std::atof(next("--hfield")); continue; }
    if (s == "--nmax") { a.n_max = std::atoi(next("--nmax")); continue; }
    if (s == "--ej") { a.E_J = std::atof(next("--ej")); continue; }
    if (s == "--ec") { a.E_C = std::atof(next("--ec")); continue; }
    if (s == "--phi") { a.phi = std::atof(next("--phi")); continue; }
    if (s == "--ng") { a.n_g = std::atof(next("--ng")); continue; }
    if (s == "--onsite") { a.onsite = next("--onsite"); continue; }
    if (s == "--j1") { a.J1 = std::atof(next("--j1")); continue; }
    if (s == "--j2") { a.J2 = std::atof(next("--j2")); continue; }
    if (s == "--j3") { a.J3 = std::atof(next("--j3")); continue; }
    if (s == "--jleg") { a.J_leg = std::atof(next("--jleg")); continue; }
    if (s == "--jrung") { a.J_rung = std::atof(next("--jrung")); continue; }
    if (s == "--delta") { a.delta = std::atof(next("--delta")); continue; }
    if (s == "--cutoff") { a.cutoff = std::atof(next("--cutoff")); continue; }
    if (s == "--tol") { a.tol = std::atof(next("--tol")); continue; }
    if (s == "--lanczos-tol") { a.lanczos_tol = std::atof(next("--lanczos-tol")); continue; }
    if (s == "--krylov") { a.krylov = std::atoi(next("--krylov")); continue; }
    if (s == "--restarts") { a.restarts = std::atoi(next("--restarts")); continue; }
    if (s == "--seed") { a.seed = std::strtoull(next("--seed"), nullptr, 10); continue; }
    if (s == "--init") { a.init = next("--init"); continue; }
    if (s == "--json") { a.json = next("--json"); continue; }
    if (s == "--single-site") { a.single_site = 1; continue; }
    if (s == "--precision") {
      const std::string v = next("--precision");
      if (v != "plain" && v != "split") { std::fprintf(stderr, "--precision takes plain or split\n"); std::exit(1); }
      a.precision = v == "split" ? 1 : 0;
      continue;
    }
    if (s == "--schedule") {
      std::stringstream ss(next("--schedule"));
      std::string tok;
      while (std::getline(ss, tok, ',')) a.schedule.push_back(std::atoi(tok.c_str()));
      continue;
    }
    if (s.size() > 1 && s[0] == '-') { std::fprintf(stderr, "Unknown flag: %s\n", s.c_str()); return 1; }
    if (pos == 0) a.L = std::atoi(s.c_str());
    else if (pos == 1) a.chi = std::atoi(s.c_str());
    else if (pos == 2) a.sweeps = std::atoi(s.c_str());
    ++pos;
  }
  if (a.L < 2 || a.chi < 1 || a.sweeps < 1) { std::fprintf(stderr, "bad L/chi/sweeps\n"); return 1; }
  try {
    if (a.model == "josephson") {
      Mpo m = josephson(a.L, a.n_max, a.E_J, a.E_C, a.n_g, a.phi, a.onsite);
      std::map<int, double> ex;
      if (a.n_max == 1 && std::fabs(a.E_J - 1.0) < 1e-10 && std::fabs(a.E_C - 0.5) < 1e-10 &&
          std::fabs(a.phi - M_PI / 4) < 1e-10 && a.n_g == 0.0)
        ex = {{4, -1.053346829927396}, {6, -1.748843818181493}};
      char extra[160];
      std::snprintf(extra, sizeof(extra), "  E_J=%.2f, E_C=%.2f, phi_ext=pi/%.1f", a.E_J, a.E_C, M_PI / a.phi);
      banner(a, "Two-Site Josephson DMRG-GPU Test (complex128)", m, extra);
      return solve(a, m, false, ex.count(a.L) ? ex[a.L] : 0.0, 1e-8, ex.count(a.L) > 0);
    } else if (a.model == "tfim") {
      Mpo m = tfim(a.L, a.J_tfim, a.h_field);
      banner(a, "Two-Site TFIM DMRG-GPU Test (float64)", m, "");
      return solve(a, m, false, 0.0, 0.0, false);
    } else if (a.model == "j1j2") {
      Mpo m = longrange(a.L, {a.J1, a.J2});
      std::map<int, double> ex;
      if (std::fabs(a.J1 - 1.0) < 1e-12 && std::fabs(a.J2 - 0.5) < 1e-12) ex = {{4, -1.5}, {6, -2.25}, {8, -3.0}};
      banner(a, "J1-J2 Heisenberg DMRG2-GPU Test (float64)", m, "");
      return solve(a, m, false, ex.count(a.L) ? ex[a.L] : 0.0, 1e-8, ex.count(a.L) > 0);
    } else if (a.model == "j1j2j3") {
      Mpo m = longrange(a.L, {a.J1, a.J2, a.J3});
      std::map<std::tuple<int, double, double, double>, double> ex = {
          {std::make_tuple(6, 1.0, 0.4, 0.2), -2.3229239173},
          {std::make_tuple(8, 1.0, 0.4, 0.2), -3.1205086380},
          {std::make_tuple(8, 1.0, 0.5, 0.25), -3.0690408638}};
      auto it = ex.find(std::make_tuple(a.L, a.J1, a.J2, a.J3));
      banner(a, "J1-J2-J3 Heisenberg DMRG2-GPU Test (float64)", m, "");
      return solve(a, m, false, it != ex.end() ? it->second : 0.0, 1e-8, it != ex.end());
    } else if (a.model == "ladder") {
      Mpo m = ladder(a.L, a.J_leg, a.J_rung);
      std::map<int, double> ex;
      if (std::fabs(a.J_leg - 1.0) < 1e-12 && std::fabs(a.J_rung - 1.0) < 1e-12)
        ex = {{2, -2.0}, {3, -3.1293852415718166}, {4, -4.2930664566945656}};
      banner(a, "Heisenberg 2-leg Ladder DMRG2-GPU Test (float64)", m, "");
      return solve(a, m, false, ex.count(a.L) ? ex[a.L] : 0.0, 1e-8, ex.count(a.L) > 0);
    } else {
      Mpo m = heisenberg(a.L, 1.0, a.delta, 0.0);
      std::map<int, double> ex;
      if (a.delta == 1.0) ex = {{4, -1.616025403784}, {8, -3.374932598688}};
      banner(a, "Two-Site Heisenberg DMRG-GPU Test (float64)", m, "");
      return solve(a, m, true, ex.count(a.L) ? ex[a.L] : 0.0, 1e-10, ex.count(a.L) > 0);
    }
  } catch (const std::exception& e) {
    std::fprintf(stderr, "ERROR: %s\n", e.what());
    return 1;
  }
}
