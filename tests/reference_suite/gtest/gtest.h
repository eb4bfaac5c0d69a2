// A small GoogleTest-compatible test harness, written for this repository (GoogleTest itself is
// not installed here). It implements the part of the GoogleTest API that the reference's CUDA
// test suites use, so those files compile unchanged against this library's headers:
//
//   TEST, TEST_F, ::testing::Test (SetUp/TearDown, RecordProperty), ::testing::Message,
//   ::testing::InitGoogleTest, RUN_ALL_TESTS, SCOPED_TRACE, ADD_FAILURE and the EXPECT_/ASSERT_
//   forms EQ, NE, LT, LE, GT, GE, TRUE, FALSE, each accepting a streamed message.
//
// Semantics follow GoogleTest's documentation: an EXPECT_ failure marks the test failed and
// continues; an ASSERT_ failure also returns from the current (void) function. Failures may be
// recorded from several threads. --gtest_filter=PATTERN[:PATTERN...] selects tests by
// "Suite.Name" with '*' and '?' wildcards; a '-' introduces patterns to exclude.
//
// Output: one "[ RUN      ]" / "[       OK ]" / "[  FAILED  ]" line per test, the failures with
// their file, line and scoped traces, and a final "[==========] N tests, P passed, F failed"
// line. The exit status is 0 when every selected test passed, 1 otherwise.
#pragma once

#include <chrono>
#include <cstdio>
#include <cstring>
#include <functional>
#include <iostream>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

namespace testing {

class Message {
  public:
    Message() = default;
    Message(const Message &other) {
        text_ << other.str();
    }
    template <typename T> Message &operator<<(const T &value) {
        text_ << value;
        return *this;
    }
    Message &operator<<(std::ostream &(*manip)(std::ostream &)) {
        text_ << manip;
        return *this;
    }
    Message &operator<<(const Message &other) {
        text_ << other.str();
        return *this;
    }
    std::string str() const {
        return text_.str();
    }

  private:
    std::ostringstream text_;
};

class Test {
  public:
    virtual ~Test() = default;
    virtual void SetUp() {}
    virtual void TearDown() {}
    virtual void TestBody() = 0;
    static void RecordProperty(const std::string &key, const std::string &value);
    static void RecordProperty(const std::string &key, long long value) {
        RecordProperty(key, std::to_string(value));
    }
};

namespace internal {

// ---- printing values in failure messages ----------------------------------------------------
template <typename T, typename = void> struct Streamable : std::false_type {};
template <typename T>
struct Streamable<T, std::void_t<decltype(std::declval<std::ostream &>() << std::declval<const T &>())>>
    : std::true_type {};
template <typename T, typename = void> struct Sized : std::false_type {};
template <typename T>
struct Sized<T, std::void_t<decltype(std::declval<const T &>().size())>> : std::true_type {};

template <typename T> std::string show(const T &value) {
    std::ostringstream out;
    if constexpr (std::is_enum_v<T>) {
        out << static_cast<long long>(static_cast<std::underlying_type_t<T>>(value));
    } else if constexpr (std::is_same_v<T, unsigned char> || std::is_same_v<T, signed char> ||
                         std::is_same_v<T, char>) {
        out << static_cast<int>(value);
    } else if constexpr (Streamable<T>::value) {
        out << value;
    } else if constexpr (Sized<T>::value) {
        out << "<container of " << value.size() << " elements>";
    } else {
        out << "<" << sizeof(T) << "-byte value>";
    }
    return out.str();
}

// ---- the run state --------------------------------------------------------------------------
struct Registered {
    std::string suite, name;
    std::function<Test *()> make;
};

struct State {
    std::mutex lock;
    std::vector<Registered> tests;
    std::vector<std::string> filters = {"*"};
    std::vector<std::string> excludes;
    bool current_failed = false;
    std::vector<std::string> traces; // outermost first
};

inline State &state() {
    static State s;
    return s;
}

inline bool register_test(const char *suite, const char *name, std::function<Test *()> make) {
    state().tests.push_back({suite, name, std::move(make)});
    return true;
}

inline void fail(const char *file, int line, const std::string &what, const std::string &note) {
    State &s = state();
    std::lock_guard<std::mutex> guard(s.lock);
    s.current_failed = true;
    std::cout << file << ":" << line << ": Failure\n" << what << "\n";
    if (!note.empty()) {
        std::cout << note << "\n";
    }
    for (auto it = s.traces.rbegin(); it != s.traces.rend(); ++it) {
        std::cout << "  trace: " << *it << "\n";
    }
    std::cout.flush();
}

// `Reporter(...) = Message() << ...` records a failure with the streamed note; operator= binds
// after every <<, so the note is complete when the failure is recorded.
class Reporter {
  public:
    Reporter(const char *file, int line, std::string what)
        : file_(file), line_(line), what_(std::move(what)) {}
    void operator=(const Message &note) const {
        fail(file_, line_, what_, note.str());
    }

  private:
    const char *file_;
    int line_;
    std::string what_;
};

// The outcome of one comparison: empty text means it held.
struct Outcome {
    bool ok = true;
    std::string text;
    explicit operator bool() const {
        return ok;
    }
};

template <typename A, typename B, typename Op>
Outcome compare(const char *op, const char *ta, const char *tb, const A &a, const B &b, Op holds) {
    if (holds(a, b)) {
        return {};
    }
    Outcome r;
    r.ok = false;
    r.text = std::string("Expected: (") + ta + ") " + op + " (" + tb + "), actual: " + show(a) +
             " vs " + show(b);
    return r;
}

inline Outcome truth(bool value, bool want, const char *text) {
    if (value == want) {
        return {};
    }
    Outcome r;
    r.ok = false;
    r.text = std::string("Value of: ") + text + "\n  Actual: " + (value ? "true" : "false") +
             "\nExpected: " + (want ? "true" : "false");
    return r;
}

class Trace {
  public:
    Trace(const char *file, int line, const Message &note) {
        State &s = state();
        std::lock_guard<std::mutex> guard(s.lock);
        s.traces.push_back(std::string(file) + ":" + std::to_string(line) + ": " + note.str());
    }
    ~Trace() {
        State &s = state();
        std::lock_guard<std::mutex> guard(s.lock);
        s.traces.pop_back();
    }
    Trace(const Trace &) = delete;
    Trace &operator=(const Trace &) = delete;
};

inline bool matches(const char *pattern, const char *text) {
    if (*pattern == '\0') return *text == '\0';
    if (*pattern == '*') return matches(pattern + 1, text) || (*text && matches(pattern, text + 1));
    if (*text == '\0') return false;
    return (*pattern == '?' || *pattern == *text) && matches(pattern + 1, text + 1);
}

inline std::vector<std::string> split(const std::string &list) {
    std::vector<std::string> out;
    std::string item;
    std::istringstream in(list);
    while (std::getline(in, item, ':')) {
        if (!item.empty()) out.push_back(item);
    }
    return out;
}

inline bool selected(const std::string &full) {
    const State &s = state();
    bool in = false;
    for (const auto &p : s.filters) in = in || matches(p.c_str(), full.c_str());
    for (const auto &p : s.excludes) in = in && !matches(p.c_str(), full.c_str());
    return in;
}

inline int run_all() {
    State &s = state();
    int run = 0, failed = 0;
    std::vector<std::string> failures;
    const auto begin = std::chrono::steady_clock::now();
    for (const Registered &t : s.tests) {
        const std::string full = t.suite + "." + t.name;
        if (!selected(full)) continue;
        ++run;
        std::cout << "[ RUN      ] " << full << std::endl;
        {
            std::lock_guard<std::mutex> guard(s.lock);
            s.current_failed = false;
        }
        const auto start = std::chrono::steady_clock::now();
        std::unique_ptr<Test> test(t.make());
        test->SetUp();
        if (!s.current_failed) test->TestBody();
        test->TearDown();
        test.reset();
        const auto ms = std::chrono::duration_cast<std::chrono::milliseconds>(
                            std::chrono::steady_clock::now() - start)
                            .count();
        if (s.current_failed) {
            ++failed;
            failures.push_back(full);
            std::cout << "[  FAILED  ] " << full << " (" << ms << " ms)" << std::endl;
        } else {
            std::cout << "[       OK ] " << full << " (" << ms << " ms)" << std::endl;
        }
    }
    const auto total = std::chrono::duration_cast<std::chrono::milliseconds>(
                           std::chrono::steady_clock::now() - begin)
                           .count();
    for (const auto &f : failures) std::cout << "[  FAILED  ] " << f << std::endl;
    std::cout << "[==========] " << run << " tests, " << run - failed << " passed, " << failed
              << " failed (" << total << " ms)" << std::endl;
    return failed == 0 ? 0 : 1;
}

} // namespace internal

inline void Test::RecordProperty(const std::string &key, const std::string &value) {
    std::lock_guard<std::mutex> guard(internal::state().lock);
    std::cout << "[ PROPERTY ] " << key << "=" << value << std::endl;
}

inline void InitGoogleTest(int *argc, char **argv) {
    internal::State &s = internal::state();
    for (int i = 1; i < *argc; ++i) {
        const char *prefix = "--gtest_filter=";
        if (std::strncmp(argv[i], prefix, std::strlen(prefix)) == 0) {
            const std::string spec = argv[i] + std::strlen(prefix);
            const auto dash = spec.find('-');
            const std::string positive = spec.substr(0, dash);
            s.filters = positive.empty() ? std::vector<std::string>{"*"}
                                         : internal::split(positive);
            s.excludes = dash == std::string::npos ? std::vector<std::string>{}
                                                   : internal::split(spec.substr(dash + 1));
        }
    }
}

} // namespace testing

#define RUN_ALL_TESTS() ::testing::internal::run_all()

#define GT_CAT_(a, b) a##b
#define GT_CAT(a, b) GT_CAT_(a, b)
#define GT_CLASS(suite, name) GT_CAT(GT_CAT(suite, _), GT_CAT(name, _Test))

#define GT_DEFINE(suite, name, base)                                                             \
    class GT_CLASS(suite, name) : public base {                                                  \
      public:                                                                                    \
        void TestBody() override;                                                                \
    };                                                                                           \
    [[maybe_unused]] static const bool GT_CAT(GT_CLASS(suite, name), _registered) =              \
        ::testing::internal::register_test(#suite, #name,                                       \
                                           [] { return new GT_CLASS(suite, name)(); });          \
    void GT_CLASS(suite, name)::TestBody()

#define TEST(suite, name) GT_DEFINE(suite, name, ::testing::Test)
#define TEST_F(fixture, name) GT_DEFINE(fixture, name, fixture)

// `switch (0) case 0: default:` keeps a dangling else after the macro from binding to it.
#define GT_CHECK(outcome, on_failure)                                                            \
    switch (0)                                                                                   \
    case 0:                                                                                      \
    default:                                                                                     \
        if (const ::testing::internal::Outcome gt_outcome = (outcome))                          \
            ;                                                                                    \
        else                                                                                     \
            on_failure ::testing::internal::Reporter(__FILE__, __LINE__, gt_outcome.text) =      \
                ::testing::Message()

#define GT_CMP(op, a, b)                                                                         \
    ::testing::internal::compare(#op, #a, #b, (a), (b),                                          \
                                 [](const auto &x, const auto &y) { return x op y; })

#define EXPECT_EQ(a, b) GT_CHECK(GT_CMP(==, a, b), )
#define EXPECT_NE(a, b) GT_CHECK(GT_CMP(!=, a, b), )
#define EXPECT_LT(a, b) GT_CHECK(GT_CMP(<, a, b), )
#define EXPECT_LE(a, b) GT_CHECK(GT_CMP(<=, a, b), )
#define EXPECT_GT(a, b) GT_CHECK(GT_CMP(>, a, b), )
#define EXPECT_GE(a, b) GT_CHECK(GT_CMP(>=, a, b), )
#define EXPECT_TRUE(c) GT_CHECK(::testing::internal::truth(static_cast<bool>(c), true, #c), )
#define EXPECT_FALSE(c) GT_CHECK(::testing::internal::truth(static_cast<bool>(c), false, #c), )
#define ASSERT_EQ(a, b) GT_CHECK(GT_CMP(==, a, b), return)
#define ASSERT_NE(a, b) GT_CHECK(GT_CMP(!=, a, b), return)
#define ASSERT_LT(a, b) GT_CHECK(GT_CMP(<, a, b), return)
#define ASSERT_LE(a, b) GT_CHECK(GT_CMP(<=, a, b), return)
#define ASSERT_GT(a, b) GT_CHECK(GT_CMP(>, a, b), return)
#define ASSERT_GE(a, b) GT_CHECK(GT_CMP(>=, a, b), return)
#define ASSERT_TRUE(c) GT_CHECK(::testing::internal::truth(static_cast<bool>(c), true, #c), return)
#define ASSERT_FALSE(c)                                                                          \
    GT_CHECK(::testing::internal::truth(static_cast<bool>(c), false, #c), return)

#define ADD_FAILURE() ::testing::internal::Reporter(__FILE__, __LINE__, "Failed") = ::testing::Message()
#define FAIL() return ADD_FAILURE()
#define SCOPED_TRACE(note)                                                                       \
    const ::testing::internal::Trace GT_CAT(gt_trace_, __LINE__)(__FILE__, __LINE__,             \
                                                                 ::testing::Message() << note)
