// Test stand-in for ChronusQ's include/cerr.hpp: CErr prints the message and
// throws std::runtime_error("FATAL"), as the reference's does.
#pragma once
#include <iostream>
#include <stdexcept>
#include <string>

namespace ChronusQ {
[[noreturn]] inline void CErr(const std::string& msg) {
  std::cerr << msg << std::endl;
  throw std::runtime_error("FATAL");
}
}  // namespace ChronusQ
