// A small gtest-compatible header (test infrastructure): enough of googletest's API to
// compile a parameterized test suite written for it -- TestWithParam / GetParam,
// TEST_P, INSTANTIATE_TEST_SUITE_P with Values and a name generator, and the
// EXPECT_/ASSERT_ comparison macros with streamed messages. The runner is
// gtest_main.cc. googletest itself is not installed in this image.
#pragma once
#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <iostream>
#include <memory>
#include <sstream>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

namespace testing {

template <class T>
struct TestParamInfo {
    T param;
    size_t index;
};

template <class T>
class TestWithParam {
  public:
    using ParamType = T;
    virtual ~TestWithParam() = default;
    virtual void TestBody() = 0;
    static const T &GetParam() { return *current(); }
    static const T *&current() {
        static const T *p = nullptr;
        return p;
    }
};

template <class First, class... Rest>
std::vector<First> Values(const First &first, const Rest &...rest) {
    return std::vector<First>{first, rest...};
}

class Message {
    std::ostringstream os_;

  public:
    template <class V>
    Message &operator<<(const V &v) {
        os_ << v;
        return *this;
    }
    std::string str() const { return os_.str(); }
};

namespace shim {

inline bool &failed() {
    static bool f = false;
    return f;
}

// non-fatal failure: reports when the full statement (with streamed text) ends
class Reporter {
    std::ostringstream os_;

  public:
    Reporter(const char *file, int line, const std::string &what) {
        os_ << file << ":" << line << ": Failure\n" << what << "\n";
        failed() = true;
    }
    template <class V>
    Reporter &operator<<(const V &v) {
        os_ << v;
        return *this;
    }
    ~Reporter() { std::cerr << os_.str() << std::endl; }
};

// fatal failure: "return AssertHelper(...) = Message() << ..." leaves the test body
struct AssertHelper {
    const char *file;
    int line;
    std::string what;
    void operator=(const Message &m) const {
        std::cerr << file << ":" << line << ": Failure\n" << what << "\n" << m.str() << std::endl;
        failed() = true;
    }
};

template <class A, class B>
std::string describe(const char *ea, const char *op, const char *eb, const A &a, const B &b) {
    std::ostringstream os;
    os << "Expected: (" << ea << ") " << op << " (" << eb << ")";
    if constexpr (std::is_arithmetic_v<A> && std::is_arithmetic_v<B>) os << ", actual: " << a << " vs " << b;
    return os.str();
}

struct Runnable {
    std::string name;
    std::function<bool()> run;
};

inline std::vector<Runnable> &runnables() {
    static std::vector<Runnable> v;
    return v;
}

// a test object is owned through its public virtual base (fixtures may keep their own
// destructor protected, as googletest allows)
template <class Fixture>
using TestPtr = std::unique_ptr<TestWithParam<typename Fixture::ParamType>>;

template <class Fixture>
std::vector<std::pair<std::string, std::function<TestPtr<Fixture>()>>> &suite() {
    static std::vector<std::pair<std::string, std::function<TestPtr<Fixture>()>>> v;
    return v;
}

template <class Fixture>
int register_test(const char *name, std::function<TestPtr<Fixture>()> make) {
    suite<Fixture>().push_back({name, make});
    return 0;
}

template <class Fixture, class Vec, class NameFn>
int instantiate(const char *prefix, const char *fixture, const Vec &values, NameFn namefn) {
    using T = typename Fixture::ParamType;
    for (size_t k = 0; k < values.size(); ++k) {
        auto param = std::make_shared<T>(values[k]);
        const std::string pname = namefn(TestParamInfo<T>{values[k], k});
        for (auto &t : suite<Fixture>()) {
            auto make = t.second;
            runnables().push_back({std::string(prefix) + "/" + fixture + "." + t.first + "/" + pname, [param, make]() {
                                       Fixture::current() = param.get();
                                       failed() = false;
                                       TestPtr<Fixture> f = make();
                                       f->TestBody();
                                       return !failed();
                                   }});
        }
    }
    return 0;
}

} // namespace shim
} // namespace testing

#define SHIM_CAT_(a, b) a##b
#define SHIM_CAT(a, b) SHIM_CAT_(a, b)

#define TEST_P(Fixture, Name)                                                                                   \
    class Fixture##_##Name##_Test : public Fixture {                                                            \
      public:                                                                                                   \
        void TestBody() override;                                                                               \
    };                                                                                                          \
    static int Fixture##_##Name##_registered =                                                                  \
        ::testing::shim::register_test<Fixture>(#Name, []() -> ::testing::shim::TestPtr<Fixture> {           \
            return ::testing::shim::TestPtr<Fixture>(new Fixture##_##Name##_Test());                             \
        });                                                                                                     \
    void Fixture##_##Name##_Test::TestBody()

#define INSTANTIATE_TEST_SUITE_P(Prefix, Fixture, ...)                                                          \
    static int SHIM_CAT(Prefix##_##Fixture##_instantiated_, __LINE__) =                                        \
        ::testing::shim::instantiate<Fixture>(#Prefix, #Fixture, __VA_ARGS__)

#define SHIM_EXPECT_(cond, text)                                                                                \
    switch (0)                                                                                                  \
    case 0:                                                                                                     \
    default:                                                                                                    \
        if (cond)                                                                                               \
            ;                                                                                                   \
        else                                                                                                    \
            ::testing::shim::Reporter(__FILE__, __LINE__, text)

#define SHIM_ASSERT_(cond, text)                                                                                \
    switch (0)                                                                                                  \
    case 0:                                                                                                     \
    default:                                                                                                    \
        if (cond)                                                                                               \
            ;                                                                                                   \
        else                                                                                                    \
            return ::testing::shim::AssertHelper{__FILE__, __LINE__, text} = ::testing::Message()

#define EXPECT_NEAR(a, b, tol)                                                                                  \
    SHIM_EXPECT_(std::fabs((double)(a) - (double)(b)) <= (double)(tol),                                         \
                 ::testing::shim::describe(#a, "near", #b, (double)(a), (double)(b)))
#define EXPECT_LT(a, b) SHIM_EXPECT_((a) < (b), ::testing::shim::describe(#a, "<", #b, (a), (b)))
#define EXPECT_NE(a, b) SHIM_EXPECT_((a) != (b), ::testing::shim::describe(#a, "!=", #b, (a), (b)))
#define EXPECT_EQ(a, b) SHIM_EXPECT_((a) == (b), ::testing::shim::describe(#a, "==", #b, (a), (b)))
#define EXPECT_TRUE(c) SHIM_EXPECT_((c), std::string("Expected true: ") + #c)
#define ASSERT_NE(a, b) SHIM_ASSERT_((a) != (b), ::testing::shim::describe(#a, "!=", #b, (a), (b)))
#define ASSERT_EQ(a, b) SHIM_ASSERT_((a) == (b), ::testing::shim::describe(#a, "==", #b, (a), (b)))
#define ASSERT_TRUE(c) SHIM_ASSERT_((c), std::string("Expected true: ") + #c)
