/*
 * poptmx.h -- stand-in for the command-line parsing library the reference
 * uses, for compiling lct.cpp without it.  Test infrastructure only.  lct.cpp
 * calls only poptmx::_conversion(float*, string) (lct.cpp:243), which parses
 * the parameter of "NAME:param" filter strings; this version parses one
 * number with strtod and accepts it only if the whole string was consumed,
 * returning 1 on success and 0 otherwise.
 */
#ifndef CTAS_ORACLE_SHIM_POPTMX_H
#define CTAS_ORACLE_SHIM_POPTMX_H

#include <cstdlib>
#include <string>

namespace poptmx {

inline int _conversion(float *val, const std::string &in) {
  if (in.empty()) return 0;
  char *end = nullptr;
  const double v = std::strtod(in.c_str(), &end);
  if (!end || *end != '\0') return 0;
  *val = (float)v;
  return 1;
}

}  // namespace poptmx

#endif
