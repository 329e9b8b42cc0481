/*
 * Minimal stand-in for GoogleTest, enough to compile and run the reference implementation's own hot-path test
 * files (tests/apsp, tests/dijkstra, tests/delta_stepping, tests/centrality) at one MPI rank through the
 * single-rank MPI shim. Supports TEST_F, TEST_P, INSTANTIATE_TEST_SUITE_P with testing::Values, GetParam,
 * ASSERT_/EXPECT_ {EQ, NE, TRUE, FALSE, NEAR, LT, LE, GT, GE, THROW}, InitGoogleTest and RUN_ALL_TESTS.
 * Test infrastructure for the oracle only.
 */
#pragma once

#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <iostream>
#include <memory>
#include <sstream>
#include <string>
#include <tuple>
#include <type_traits>
#include <utility>
#include <vector>

namespace testing {

class Test {
public:
    virtual ~Test() = default;
    virtual void SetUp() { }
    virtual void TearDown() { }
    virtual void TestBody() = 0;
};

template <typename T>
class WithParamInterface {
public:
    using ParamType = T;
    virtual ~WithParamInterface() = default;
    [[nodiscard]] static const T& GetParam() { return *current_parameter; }
    inline static const T* current_parameter = nullptr;
};

template <typename T>
struct TestParamInfo {
    T param;
    std::size_t index;
};

template <typename... Ts>
struct ValueArray {
    std::tuple<Ts...> values;

    template <typename T>
    [[nodiscard]] std::vector<T> to_vector() const {
        return std::apply([](const auto&... v) { return std::vector<T>{ static_cast<T>(v)... }; }, values);
    }
};

template <typename... Ts>
[[nodiscard]] ValueArray<Ts...> Values(Ts... values) {
    return { std::tuple<Ts...>{ values... } };
}

namespace internal {

struct Registry {
    struct Plain {
        std::string suite;
        std::string name;
        std::function<std::unique_ptr<Test>()> factory;
    };
    struct Parameterised {
        std::string suite;
        std::string name;
        std::function<void(std::size_t)> run; /* runs the test body for the instantiation's value with this index */
        std::function<std::size_t()> count;
    };

    std::vector<Plain> plain{};
    std::vector<Parameterised> parameterised{};
    int failures_in_current_test = 0;
    int failed_tests = 0;
    int passed_tests = 0;

    static Registry& get() {
        static Registry registry;
        return registry;
    }
};

/* The values of every instantiation of a parameterised fixture, in registration order. */
template <typename Fixture>
std::vector<typename Fixture::ParamType>& instantiated_values() {
    static std::vector<typename Fixture::ParamType> values;
    return values;
}

template <typename Fixture, typename Generator>
int register_instantiation(const Generator& generator) {
    auto values = generator.template to_vector<typename Fixture::ParamType>();
    auto& all = instantiated_values<Fixture>();
    all.insert(all.end(), values.begin(), values.end());
    return 0;
}

template <typename Fixture, typename Generator, typename Namer>
int register_instantiation(const Generator& generator, const Namer&) {
    return register_instantiation<Fixture>(generator);
}

inline void run_one(Test& test) {
    test.SetUp();
    test.TestBody();
    test.TearDown();
}

template <typename Fixture, typename TestClass>
int register_parameterised(const char* suite, const char* name) {
    Registry::get().parameterised.push_back({ suite, name,
                                              [](std::size_t index) {
                                                  const auto& values = instantiated_values<Fixture>();
                                                  Fixture::current_parameter = &values[index];
                                                  auto test = TestClass{};
                                                  run_one(test);
                                              },
                                              [] { return instantiated_values<Fixture>().size(); } });
    return 0;
}

template <typename TestClass>
int register_plain(const char* suite, const char* name) {
    Registry::get().plain.push_back({ suite, name, [] { return std::unique_ptr<Test>(new TestClass()); } });
    return 0;
}

template <typename T, typename = void>
struct printable : std::false_type { };
template <typename T>
struct printable<T, std::void_t<decltype(std::declval<std::ostream&>() << std::declval<const T&>())>> : std::true_type { };

template <typename T>
std::string show(const T& value) {
    if constexpr (printable<T>::value) {
        auto out = std::ostringstream{};
        out.precision(17);
        out << value;
        return out.str();
    } else {
        return "<unprintable>";
    }
}

inline void report(const char* file, int line, const std::string& what) {
    std::fprintf(stderr, "%s:%d: Failure\n%s\n", file, line, what.c_str());
    ++Registry::get().failures_in_current_test;
}

template <typename A, typename B>
bool check_eq(const A& a, const B& b, const char* ea, const char* eb, const char* file, int line) {
    if constexpr (std::is_integral_v<A> && std::is_integral_v<B>) {
        if (std::cmp_equal(a, b)) {
            return true;
        }
    } else {
        if (a == b) {
            return true;
        }
    }
    report(file, line, std::string("Expected equality of ") + ea + " (" + show(a) + ") and " + eb + " (" + show(b) + ")");
    return false;
}

inline bool check_near(double a, double b, double tolerance, const char* ea, const char* eb, const char* file, int line) {
    if (std::fabs(a - b) <= tolerance) {
        return true;
    }
    report(file, line, std::string("The difference between ") + ea + " (" + show(a) + ") and " + eb + " (" + show(b) + ") exceeds " + show(tolerance));
    return false;
}

inline bool check_true(bool value, const char* expression, bool expected, const char* file, int line) {
    if (value == expected) {
        return true;
    }
    report(file, line, std::string("Value of ") + expression + " is " + (value ? "true" : "false"));
    return false;
}

template <typename A, typename B, typename Compare>
bool check_cmp(const A& a, const B& b, Compare compare, const char* op, const char* ea, const char* eb, const char* file, int line) {
    if (compare(a, b)) {
        return true;
    }
    report(file, line, std::string("Expected ") + ea + " " + op + " " + eb + " (" + show(a) + " vs " + show(b) + ")");
    return false;
}

} // namespace internal

inline void InitGoogleTest(int*, char**) { }

} // namespace testing

inline int RUN_ALL_TESTS() {
    auto& registry = testing::internal::Registry::get();
    const char* filter = std::getenv("GTEST_SHIM_FILTER");
    const auto run = [&](const std::string& label, const std::function<void()>& body) {
        if (filter != nullptr && label.find(filter) == std::string::npos) {
            return;
        }
        registry.failures_in_current_test = 0;
        try {
            body();
        } catch (const std::exception& e) {
            std::fprintf(stderr, "%s: unexpected exception: %s\n", label.c_str(), e.what());
            ++registry.failures_in_current_test;
        }
        if (registry.failures_in_current_test == 0) {
            ++registry.passed_tests;
            std::printf("[       OK ] %s\n", label.c_str());
        } else {
            ++registry.failed_tests;
            std::printf("[  FAILED  ] %s\n", label.c_str());
        }
    };
    for (const auto& test : registry.plain) {
        run(test.suite + "." + test.name, [&] {
            auto instance = test.factory();
            testing::internal::run_one(*instance);
        });
    }
    for (const auto& test : registry.parameterised) {
        const auto count = test.count();
        for (std::size_t i = 0; i < count; ++i) {
            run(test.suite + "." + test.name + "/" + std::to_string(i), [&] { test.run(i); });
        }
    }
    std::printf("[==========] %d passed, %d failed\n", registry.passed_tests, registry.failed_tests);
    return registry.failed_tests == 0 ? 0 : 1;
}

#define GTEST_SHIM_CLASS_(fixture, name) fixture##_##name##_Test

#define TEST_F(fixture, name)                                                                                                                                 \
    class GTEST_SHIM_CLASS_(fixture, name) : public fixture {                                                                                                 \
    public:                                                                                                                                                    \
        void TestBody() override;                                                                                                                             \
    };                                                                                                                                                         \
    [[maybe_unused]] static const int gtest_shim_registered_##fixture##_##name =                                                                              \
        ::testing::internal::register_plain<GTEST_SHIM_CLASS_(fixture, name)>(#fixture, #name);                                                              \
    void GTEST_SHIM_CLASS_(fixture, name)::TestBody()

#define TEST_P(fixture, name)                                                                                                                                 \
    class GTEST_SHIM_CLASS_(fixture, name) : public fixture {                                                                                                 \
    public:                                                                                                                                                    \
        void TestBody() override;                                                                                                                             \
    };                                                                                                                                                         \
    [[maybe_unused]] static const int gtest_shim_registered_##fixture##_##name =                                                                              \
        ::testing::internal::register_parameterised<fixture, GTEST_SHIM_CLASS_(fixture, name)>(#fixture, #name);                                            \
    void GTEST_SHIM_CLASS_(fixture, name)::TestBody()

#define INSTANTIATE_TEST_SUITE_P(prefix, fixture, ...)                                                                                                        \
    [[maybe_unused]] static const int gtest_shim_instantiated_##prefix##_##fixture = ::testing::internal::register_instantiation<fixture>(__VA_ARGS__)

namespace testing {
/* Collects the text streamed after a failed assertion ("ASSERT_EQ(a, b) << details"). */
class Message {
public:
    template <typename T>
    Message& operator<<(const T& value) {
        stream_ << internal::show(value);
        return *this;
    }
    [[nodiscard]] std::string str() const { return stream_.str(); }

private:
    std::ostringstream stream_{};
};
namespace internal {
struct AssertHelper {
    void operator=(const Message& message) const {
        const auto text = message.str();
        if (!text.empty()) {
            std::fprintf(stderr, "  %s\n", text.c_str());
        }
    }
};
} // namespace internal
} // namespace testing

#define GTEST_SHIM_ASSERT_(condition)                                                                                                                         \
    if (condition)                                                                                                                                             \
        ;                                                                                                                                                      \
    else                                                                                                                                                       \
        return ::testing::internal::AssertHelper() = ::testing::Message()

#define GTEST_SHIM_EXPECT_(condition)                                                                                                                         \
    if (condition)                                                                                                                                             \
        ;                                                                                                                                                      \
    else                                                                                                                                                       \
        ::testing::internal::AssertHelper() = ::testing::Message()

#define ASSERT_EQ(a, b) GTEST_SHIM_ASSERT_(::testing::internal::check_eq((a), (b), #a, #b, __FILE__, __LINE__))
#define EXPECT_EQ(a, b) GTEST_SHIM_EXPECT_(::testing::internal::check_eq((a), (b), #a, #b, __FILE__, __LINE__))
#define ASSERT_NE(a, b) GTEST_SHIM_ASSERT_(::testing::internal::check_cmp((a), (b), [](const auto& x, const auto& y) { return !(x == y); }, "!=", #a, #b, __FILE__, __LINE__))
#define EXPECT_NE(a, b) GTEST_SHIM_EXPECT_(::testing::internal::check_cmp((a), (b), [](const auto& x, const auto& y) { return !(x == y); }, "!=", #a, #b, __FILE__, __LINE__))
#define ASSERT_LT(a, b) GTEST_SHIM_ASSERT_(::testing::internal::check_cmp((a), (b), [](const auto& x, const auto& y) { return x < y; }, "<", #a, #b, __FILE__, __LINE__))
#define ASSERT_LE(a, b) GTEST_SHIM_ASSERT_(::testing::internal::check_cmp((a), (b), [](const auto& x, const auto& y) { return x <= y; }, "<=", #a, #b, __FILE__, __LINE__))
#define ASSERT_GT(a, b) GTEST_SHIM_ASSERT_(::testing::internal::check_cmp((a), (b), [](const auto& x, const auto& y) { return x > y; }, ">", #a, #b, __FILE__, __LINE__))
#define ASSERT_GE(a, b) GTEST_SHIM_ASSERT_(::testing::internal::check_cmp((a), (b), [](const auto& x, const auto& y) { return x >= y; }, ">=", #a, #b, __FILE__, __LINE__))
#define EXPECT_LT(a, b) GTEST_SHIM_EXPECT_(::testing::internal::check_cmp((a), (b), [](const auto& x, const auto& y) { return x < y; }, "<", #a, #b, __FILE__, __LINE__))
#define EXPECT_LE(a, b) GTEST_SHIM_EXPECT_(::testing::internal::check_cmp((a), (b), [](const auto& x, const auto& y) { return x <= y; }, "<=", #a, #b, __FILE__, __LINE__))
#define EXPECT_GT(a, b) GTEST_SHIM_EXPECT_(::testing::internal::check_cmp((a), (b), [](const auto& x, const auto& y) { return x > y; }, ">", #a, #b, __FILE__, __LINE__))
#define EXPECT_GE(a, b) GTEST_SHIM_EXPECT_(::testing::internal::check_cmp((a), (b), [](const auto& x, const auto& y) { return x >= y; }, ">=", #a, #b, __FILE__, __LINE__))
#define ASSERT_NEAR(a, b, tol) GTEST_SHIM_ASSERT_(::testing::internal::check_near((a), (b), (tol), #a, #b, __FILE__, __LINE__))
#define EXPECT_NEAR(a, b, tol) GTEST_SHIM_EXPECT_(::testing::internal::check_near((a), (b), (tol), #a, #b, __FILE__, __LINE__))
#define ASSERT_DOUBLE_EQ(a, b) ASSERT_NEAR((a), (b), 4 * 2.220446049250313e-16 * std::fabs(static_cast<double>(b)))
#define EXPECT_DOUBLE_EQ(a, b) EXPECT_NEAR((a), (b), 4 * 2.220446049250313e-16 * std::fabs(static_cast<double>(b)))
#define ASSERT_TRUE(c) GTEST_SHIM_ASSERT_(::testing::internal::check_true(static_cast<bool>(c), #c, true, __FILE__, __LINE__))
#define EXPECT_TRUE(c) GTEST_SHIM_EXPECT_(::testing::internal::check_true(static_cast<bool>(c), #c, true, __FILE__, __LINE__))
#define ASSERT_FALSE(c) GTEST_SHIM_ASSERT_(::testing::internal::check_true(static_cast<bool>(c), #c, false, __FILE__, __LINE__))
#define EXPECT_FALSE(c) GTEST_SHIM_EXPECT_(::testing::internal::check_true(static_cast<bool>(c), #c, false, __FILE__, __LINE__))

#define GTEST_SHIM_THROWS_(statement, exception_type, on_fail)                                                                                               \
    {                                                                                                                                                          \
        bool gtest_shim_caught = false;                                                                                                                       \
        try {                                                                                                                                                  \
            statement;                                                                                                                                         \
        } catch (const exception_type&) {                                                                                                                     \
            gtest_shim_caught = true;                                                                                                                          \
        } catch (...) {                                                                                                                                        \
        }                                                                                                                                                      \
        if (!gtest_shim_caught) {                                                                                                                              \
            ::testing::internal::report(__FILE__, __LINE__, "Expected " #statement " to throw " #exception_type);                                            \
            on_fail;                                                                                                                                           \
        }                                                                                                                                                      \
    }
#define ASSERT_THROW(statement, exception_type) GTEST_SHIM_THROWS_(statement, exception_type, return)
#define EXPECT_THROW(statement, exception_type) GTEST_SHIM_THROWS_(statement, exception_type, (void)0)
#define ASSERT_ANY_THROW(statement) GTEST_SHIM_THROWS_(statement, std::exception, return)
#define ASSERT_NO_THROW(statement) statement
#define EXPECT_NO_THROW(statement) statement
