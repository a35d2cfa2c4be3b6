// A minimal stand-in for googletest, enough to run the reference's unit-test
// sources against the oracle: TEST registers a function, EXPECT_* / ASSERT_*
// record every evaluated comparison by source line (an ASSERT does not
// abort the test here; every expectation is evaluated and recorded).
#pragma once
#include <cstdio>
#include <cmath>
#include <map>
#include <string>
#include <vector>

namespace rt {

struct Case {
  const char* suite;
  const char* name;
  void (*fn)();
};

inline std::vector<Case>& registry() {
  static std::vector<Case> r;
  return r;
}

struct Reg {
  Reg(const char* s, const char* n, void (*f)()) { registry().push_back({s, n, f}); }
};

// Per source line: how many times it was evaluated and how many failed, with
// the operands of the first failure.
struct LineStat {
  long long evaluated = 0, failed = 0;
  double a = 0, b = 0;
  std::string kind;
};

struct State {
  std::string test;
  std::map<std::pair<std::string, int>, LineStat> lines;
};

inline State& state() {
  static State s;
  return s;
}

// Lets `EXPECT_LT(a, b) << "message";` compile; the message is dropped.
struct Msg {
  template <class T> Msg& operator<<(const T&) { return *this; }
};

inline Msg record(int line, bool ok, const char* kind, double a, double b) {
  LineStat& st = state().lines[{state().test, line}];
  st.kind = kind;
  st.evaluated += 1;
  if (!ok) {
    if (st.failed == 0) { st.a = a; st.b = b; }
    st.failed += 1;
  }
  return Msg{};
}

}  // namespace rt

#define RT_CAT2(a, b) a##b
#define RT_CAT(a, b) RT_CAT2(a, b)
#define TEST(S, N)                                                   \
  static void RT_CAT(rt_fn_, RT_CAT(S, RT_CAT(_, N)))();             \
  static rt::Reg RT_CAT(rt_reg_, RT_CAT(S, RT_CAT(_, N)))(#S, #N,    \
                                                  RT_CAT(rt_fn_, RT_CAT(S, RT_CAT(_, N)))); \
  static void RT_CAT(rt_fn_, RT_CAT(S, RT_CAT(_, N)))()

#define RT_CMP(a, b, op, kind)                                                             \
  ([&]() -> rt::Msg {                                                                    \
    auto rt_a = (a);                                                                     \
    auto rt_b = (b);                                                                     \
    return rt::record(__LINE__, rt_a op rt_b, kind, (double)rt_a, (double)rt_b);         \
  }())
#define EXPECT_LT(a, b) RT_CMP(a, b, <, "LT")
#define EXPECT_LE(a, b) RT_CMP(a, b, <=, "LE")
#define EXPECT_GT(a, b) RT_CMP(a, b, >, "GT")
#define EXPECT_GE(a, b) RT_CMP(a, b, >=, "GE")
#define EXPECT_EQ(a, b) RT_CMP(a, b, ==, "EQ")
#define EXPECT_NE(a, b) RT_CMP(a, b, !=, "NE")
#define EXPECT_FLOAT_EQ(a, b) RT_CMP((float)(a), (float)(b), ==, "EQ")
#define EXPECT_DOUBLE_EQ(a, b) RT_CMP((double)(a), (double)(b), ==, "EQ")
#define EXPECT_NEAR(a, b, e)                                                               \
  ([&]() -> rt::Msg {                                                                    \
    double rt_a = (double)(a), rt_b = (double)(b);                                       \
    return rt::record(__LINE__, std::fabs(rt_a - rt_b) <= (double)(e), "NEAR", rt_a, rt_b); \
  }())
#define EXPECT_TRUE(c) rt::record(__LINE__, (bool)(c), "TRUE", 0, 0)
#define EXPECT_FALSE(c) rt::record(__LINE__, !(bool)(c), "FALSE", 0, 0)
#define ASSERT_LT EXPECT_LT
#define ASSERT_LE EXPECT_LE
#define ASSERT_GT EXPECT_GT
#define ASSERT_GE EXPECT_GE
#define ASSERT_EQ EXPECT_EQ
#define ASSERT_NE EXPECT_NE
#define ASSERT_NEAR EXPECT_NEAR
#define ASSERT_TRUE EXPECT_TRUE
#define ASSERT_FALSE EXPECT_FALSE
