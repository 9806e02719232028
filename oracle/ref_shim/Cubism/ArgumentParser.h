// Stand-in (oracle test infrastructure): the command-line parser the
// reference's obstacle constructors accept; this build constructs obstacles
// from ObstacleArguments, so every lookup returns its default.
#pragma once
#include <string>

#include "core.h"

namespace cubism {
class ArgumentParser {
 public:
  struct Value {
    double asDouble(double d = 0) const { return d; }
    int asInt(int d = 0) const { return d; }
    bool asBool(bool d = false) const { return d; }
    std::string asString(const std::string& d = "") const { return d; }
  };
  Value operator()(const std::string&) const { return Value{}; }
  bool check(const std::string&) const { return false; }
};
}  // namespace cubism
