#pragma once
#include <stddef.h>
#include <string>
#include <vector>

#include "lsg_mech.h"

namespace lsg {

struct HostMech {
  MechLayout layout;
  std::vector<unsigned char> buffer;   // flattened [double region][int region]
  std::vector<std::string> species;
  std::vector<double> mw;
  bool has_transport = false;          // the blob carries tr_* fits
  TransportLayout tlayout{};
  std::vector<unsigned char> tbuffer;  // flattened transport table
  std::vector<int> iteta;              // light species with thermal-diffusion ratios
};

bool build_mechanism(const void* blob, size_t nbytes, HostMech& out, std::string& err);

}  // namespace lsg
