// Hamiltonian MPO builders for the CLI (host code).
//
// Same models as the reference driver (gpu-rocm/dmrg2-gpu/src/test_dmrg2_gpu.cpp:20-191,
// gpu-rocm/common/challenge_mpos.h:50-360), written in the row-major layout of
// include/dmrg2_b200.h: W[i] has shape (Dl, Dr, d, d) with axes
// (mpo_l, mpo_r, s_in, s_out) and Dl_0 = Dr_{L-1} = 1.
#pragma once

#include <string>
#include <vector>

namespace dmrg2cli {

struct Mpo {
  int L = 0, d = 0;
  bool cplx = false;
  std::vector<int> Dl, Dr;
  std::vector<std::vector<double>> W;  // complex: interleaved (re, im)
  std::string name;
};

Mpo heisenberg(int L, double J, double delta, double hz);
Mpo tfim(int L, double J, double h);
// onsite: "reference" -> E_C n^2 - n_g n ; "shifted" -> E_C (n - n_g)^2
Mpo josephson(int L, int n_max, double E_J, double E_C, double n_g, double phi,
              const std::string& onsite);
Mpo longrange(int L, const std::vector<double>& Js);  // J1-J2 (2 terms), J1-J2-J3 (3 terms)
Mpo ladder(int L_rungs, double J_leg, double J_rung);

}  // namespace dmrg2cli
