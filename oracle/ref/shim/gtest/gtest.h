// Stand-in for googletest, enough for the reference's common/testHao/
// gtest_custom.h to compile when its library sources are built for the CPU
// baseline (the reference's own tests are not built).  Part of the
// oracle's reference build (test infrastructure only).
#pragma once
namespace testing {
class AssertionResult {
public:
    explicit AssertionResult(bool ok = true) : ok_(ok) {}
    template <class T>
    AssertionResult &operator<<(const T &) { return *this; }
    explicit operator bool() const { return ok_; }

private:
    bool ok_;
};
inline AssertionResult AssertionSuccess() { return AssertionResult(true); }
inline AssertionResult AssertionFailure() { return AssertionResult(false); }
}  // namespace testing
#define EXPECT_TRUE(x) ((void)(x))
#define EXPECT_FALSE(x) ((void)(x))
#define EXPECT_EQ(a, b) ((void)(a), (void)(b))
#define EXPECT_NEAR(a, b, c) ((void)(a), (void)(b), (void)(c))
#define EXPECT_DOUBLE_EQ(a, b) ((void)(a), (void)(b))
#define EXPECT_FLOAT_EQ(a, b) ((void)(a), (void)(b))
