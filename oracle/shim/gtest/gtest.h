// Tiny stand-in for googletest so the reference's own test file can run
// against the reference build (test infrastructure only).
#ifndef ORACLE_SHIM_GTEST_H_
#define ORACLE_SHIM_GTEST_H_
#include <cstdio>
#include <cstring>
#include <functional>
#include <string>
#include <vector>
namespace shimtest {
struct Case { std::string name; std::function<void()> fn; };
inline std::vector<Case>& registry() { static std::vector<Case> r; return r; }
inline int& failures() { static int f = 0; return f; }
struct Reg { Reg(const char* n, std::function<void()> f) { registry().push_back({n, f}); } };
}  // namespace shimtest
#define TEST(suite, name)                                                   \
  static void suite##_##name##_body();                                      \
  static shimtest::Reg suite##_##name##_reg(#suite "." #name,               \
                                            suite##_##name##_body);         \
  static void suite##_##name##_body()
#define SHIM_CHECK_LE(a, b, fatal)                                          \
  do {                                                                      \
    double sa_ = (a), sb_ = (b);                                            \
    std::printf("    value %.6e  bound %.6e  %s\n", sa_, sb_,               \
                sa_ <= sb_ ? "ok" : "FAIL");                                \
    if (!(sa_ <= sb_)) { shimtest::failures()++; if (fatal) return; }       \
  } while (0)
#define EXPECT_LE(a, b) SHIM_CHECK_LE(a, b, false)
#define ASSERT_LE(a, b) SHIM_CHECK_LE(a, b, true)
#endif
