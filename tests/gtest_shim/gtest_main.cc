// Runner of the gtest-compatible header: every instantiated test, gtest-style report,
// exit status 1 when any failed.
#include <chrono>

#include "gtest/gtest.h"

int main() {
    auto &tests = testing::shim::runnables();
    int failed = 0;
    std::printf("[==========] Running %zu tests.\n", tests.size());
    for (auto &t : tests) {
        std::printf("[ RUN      ] %s\n", t.name.c_str());
        std::fflush(stdout);
        const auto t0 = std::chrono::steady_clock::now();
        const bool ok = t.run();
        const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        std::printf("%s %s (%.0f ms)\n", ok ? "[       OK ]" : "[  FAILED  ]", t.name.c_str(), ms);
        if (!ok) ++failed;
    }
    std::printf("[==========] %zu tests ran. %s %zu, failed %d.\n", tests.size(), "[  PASSED  ]", tests.size() - failed,
                failed);
    return failed ? 1 : 0;
}
