// Minimal googletest-compatible shim (TEST, EXPECT_TRUE/FALSE/EQ/NEAR,
// EXPECT_DEBUG_DEATH, InitGoogleTest, RUN_ALL_TESTS) used to build the
// reference's own unit tests without googletest, which is not available
// offline.  Test infrastructure only.
#pragma once

#include <cmath>
#include <cstdio>
#include <functional>
#include <string>
#include <vector>

namespace shim {

struct Case {
  const char* suite;
  const char* name;
  std::function<void()> fn;
};

inline std::vector<Case>& registry() {
  static std::vector<Case> r;
  return r;
}
inline long& n_checks() { static long n = 0; return n; }
inline long& n_fail() { static long n = 0; return n; }
inline long& n_skipped() { static long n = 0; return n; }
inline bool& case_failed() { static bool f = false; return f; }

struct Registrar {
  Registrar(const char* s, const char* n, std::function<void()> f) {
    registry().push_back({s, n, std::move(f)});
  }
};

inline void check(bool ok, const char* expr, const char* file, int line) {
  ++n_checks();
  if (!ok) {
    ++n_fail();
    case_failed() = true;
    std::printf("FAILED %s:%d: %s\n", file, line, expr);
  }
}

inline int run_all() {
  int failed_cases = 0;
  for (auto& c : registry()) {
    case_failed() = false;
    c.fn();
    if (case_failed()) {
      ++failed_cases;
      std::printf("[  FAILED  ] %s.%s\n", c.suite, c.name);
    }
  }
  std::printf("[==========] %zu tests, %d failed; %ld checks, %ld failed, %ld death checks skipped\n",
              registry().size(), failed_cases, n_checks(), n_fail(), n_skipped());
  return failed_cases ? 1 : 0;
}

}  // namespace shim

namespace testing {
inline void InitGoogleTest(int*, char**) {}
}  // namespace testing

#define RUN_ALL_TESTS() ::shim::run_all()

#define SHIM_CAT2(a, b) a##b
#define SHIM_CAT(a, b) SHIM_CAT2(a, b)
#define TEST(suite, name)                                                     \
  static void SHIM_CAT(shim_test_, SHIM_CAT(suite, name))();                  \
  static ::shim::Registrar SHIM_CAT(shim_reg_, SHIM_CAT(suite, name))(        \
      #suite, #name, &SHIM_CAT(shim_test_, SHIM_CAT(suite, name)));           \
  static void SHIM_CAT(shim_test_, SHIM_CAT(suite, name))()

#define EXPECT_TRUE(x) ::shim::check(static_cast<bool>(x), #x, __FILE__, __LINE__)
#define EXPECT_FALSE(x) ::shim::check(!static_cast<bool>(x), "!(" #x ")", __FILE__, __LINE__)
#define EXPECT_EQ(a, b) ::shim::check((a) == (b), #a " == " #b, __FILE__, __LINE__)
#define EXPECT_NEAR(a, b, tol) \
  ::shim::check(std::abs((a) - (b)) <= (tol), "|" #a " - " #b "| <= " #tol, __FILE__, __LINE__)
#define EXPECT_DEBUG_DEATH(stmt, re) (void)(++::shim::n_skipped())
