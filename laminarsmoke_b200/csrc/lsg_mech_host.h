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
};

bool build_mechanism(const void* blob, size_t nbytes, HostMech& out, std::string& err);

}  // namespace lsg
