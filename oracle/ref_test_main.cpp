// Runner for the reference's own gtest file through oracle/shim/gtest/gtest.h.
// Usage: ref_tests [substring ...] -- runs the cases whose name contains any
// substring (all cases when none given).  Test infrastructure only.
#include <cstdio>
#include <cstring>
#include "gtest/gtest.h"

int main(int argc, char** argv) {
  int ran = 0;
  for (auto& c : shimtest::registry()) {
    bool pick = argc < 2;
    for (int i = 1; i < argc; i++) {
      if (std::strstr(c.name.c_str(), argv[i])) pick = true;
    }
    if (!pick) continue;
    std::printf("[ RUN ] %s\n", c.name.c_str());
    std::fflush(stdout);
    c.fn();
    ran++;
  }
  std::printf("ran %d cases, %d failed checks\n", ran, shimtest::failures());
  return shimtest::failures() == 0 ? 0 : 1;
}
