// A minimal test framework with the names the reference's test file uses
// (::testing::Test, TEST_F, ASSERT_NEAR / ASSERT_GE / ASSERT_LT with
// streamed messages), so that file compiles unchanged against this
// library's drop-in headers (include/phi/).  Test harness only: built by
// tests/refsuite/Makefile, run by tests/test_gpu_reference_suite.py.
//
// The reference's own headers put namespace std in scope for its test file
// (hierarchy_node.h:6, included through its hierarchy_integrator.h); this
// header does the same for it, after the library's headers.
#ifndef PHI_REFSUITE_GUNIT_H_
#define PHI_REFSUITE_GUNIT_H_

#include <cmath>
#include <functional>
#include <iostream>
#include <sstream>
#include <string>
#include <utility>
#include <vector>

using namespace std;

namespace testing {

class Test {
 public:
  virtual ~Test() {}
  virtual void SetUp() {}
  virtual void TearDown() {}
  virtual void TestBody() = 0;
};

// Registered tests, in file order.
inline std::vector<std::pair<std::string, std::function<Test *()>>> &Registry() {
  static std::vector<std::pair<std::string, std::function<Test *()>>> r;
  return r;
}

inline bool Register(const char *name, std::function<Test *()> make) {
  Registry().emplace_back(name, std::move(make));
  return true;
}

// Failures of the test that is running.
inline std::vector<std::string> &Failures() {
  static std::vector<std::string> f;
  return f;
}

class Message {
 public:
  template <class T>
  Message &operator<<(const T &v) {
    ss_ << v;
    return *this;
  }
  std::string str() const { return ss_.str(); }

 private:
  std::ostringstream ss_;
};

// `return AssertHelper(...) = Message() << ...;` records the failure and
// leaves the enclosing function, as a failed ASSERT_* does.
class AssertHelper {
 public:
  AssertHelper(const char *file, int line, std::string what) : file_(file), line_(line), what_(std::move(what)) {}
  void operator=(const Message &m) const {
    std::ostringstream ss;
    ss << file_ << ":" << line_ << ": " << what_;
    const std::string extra = m.str();
    if (!extra.empty()) ss << "\n" << extra;
    Failures().push_back(ss.str());
  }

 private:
  const char *file_;
  int line_;
  std::string what_;
};

inline std::string NearText(double a, double b, double tol, const char *ea, const char *eb) {
  std::ostringstream ss;
  ss.precision(17);
  ss << "|" << ea << " - " << eb << "| = |" << a << " - " << b << "| > " << tol;
  return ss.str();
}

template <class A, class B>
std::string CmpText(const A &a, const B &b, const char *op, const char *ea, const char *eb) {
  std::ostringstream ss;
  ss.precision(17);
  ss << "expected " << ea << " " << op << " " << eb << ", got " << a << " vs " << b;
  return ss.str();
}

}  // namespace testing

#define TEST_F(Fixture, Name)                                                              \
  class Fixture##_##Name##_Test : public Fixture {                                         \
   public:                                                                                 \
    void TestBody() override;                                                              \
  };                                                                                       \
  static const bool Fixture##_##Name##_registered =                                        \
      ::testing::Register(#Fixture "." #Name, []() -> ::testing::Test * {                   \
        return new Fixture##_##Name##_Test;                                                \
      });                                                                                  \
  void Fixture##_##Name##_Test::TestBody()

#define PHI_REFSUITE_ASSERT_(ok, text) \
  if (ok)                              \
    ;                                  \
  else                                 \
    return ::testing::AssertHelper(__FILE__, __LINE__, (text)) = ::testing::Message()

#define ASSERT_NEAR(a, b, tol)                                                                  \
  PHI_REFSUITE_ASSERT_(std::fabs((double)(a) - (double)(b)) <= (double)(tol),                   \
                       ::testing::NearText((double)(a), (double)(b), (double)(tol), #a, #b))
#define ASSERT_GE(a, b) PHI_REFSUITE_ASSERT_((a) >= (b), ::testing::CmpText((a), (b), ">=", #a, #b))
#define ASSERT_LT(a, b) PHI_REFSUITE_ASSERT_((a) < (b), ::testing::CmpText((a), (b), "<", #a, #b))

#endif  // PHI_REFSUITE_GUNIT_H_
