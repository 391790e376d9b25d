// Stand-in declarations for the OpenWQ library, whose source is not vendored
// with the FLUXOS reference (src/openwq/openwq is an absent submodule).
// TEST INFRASTRUCTURE ONLY: they exist so that src/fluxos/main.cpp and
// src/fluxos/common.cpp compile for the CPU oracle. Every OpenWQ branch in the
// reference is gated on the OPENWQ module flag, which the oracle never sets.
#ifndef FLUXOS_ORACLE_OPENWQ_STUB
#define FLUXOS_ORACLE_OPENWQ_STUB
#include <armadillo>
#include <ctime>
#include <memory>
#include <string>
#include <vector>

class OpenWQ_couplercalls {};
class OpenWQ_hostModelconfig {};
class OpenWQ_json {};
class OpenWQ_wqconfig {
 public:
  int BGC_general_num_chem = 0;
  std::vector<unsigned int> BGC_general_mobile_species;
};
class OpenWQ_units {};
class OpenWQ_utils {};
class OpenWQ_readjson {};
class OpenWQ_vars {
 public:
  OpenWQ_vars(int, int) : chemass(new arma::field<arma::field<arma::Cube<double>>>(1)) {}
  std::unique_ptr<arma::field<arma::field<arma::Cube<double>>>> chemass;
};
class OpenWQ_initiate {};
class OpenWQ_watertransp {};
class OpenWQ_chem {};
class OpenWQ_extwatflux_ss {};
class OpenWQ_solver {};
class OpenWQ_output {};
#endif
