// Runner for the reference's test file compiled against this library:
// runs every registered test (or those whose names contain argv[1]) and
// prints one line per test, "PASS <name>" or "FAIL <name>" followed by the
// recorded failures, then "SUMMARY <passed> <failed>".  Exit status: 0 when
// every test ran to the end (failures are reported, not signalled).
#include <cstdio>
#include <cstring>
#include <exception>
#include <iostream>

#include "testing/base/public/gunit.h"

int main(int argc, char **argv) {
  const char *filter = argc > 1 ? argv[1] : nullptr;
  int passed = 0, failed = 0;
  for (auto &entry : ::testing::Registry()) {
    if (filter && !std::strstr(entry.first.c_str(), filter)) continue;
    ::testing::Failures().clear();
    ::testing::Test *t = entry.second();
    try {
      t->SetUp();
      t->TestBody();
      t->TearDown();
    } catch (const std::exception &e) {
      ::testing::Failures().push_back(std::string("exception: ") + e.what());
    }
    delete t;
    const bool ok = ::testing::Failures().empty();
    std::cout << (ok ? "PASS " : "FAIL ") << entry.first << "\n";
    for (const auto &f : ::testing::Failures()) std::cout << "  " << f << "\n";
    std::cout.flush();
    (ok ? passed : failed) += 1;
  }
  std::cout << "SUMMARY " << passed << " " << failed << std::endl;
  return 0;
}
