// Runs every TEST registered by one of the reference's unit-test sources
// (compiled against shim/refapi.h, which restates the reference's API over
// the oracle) and writes one JSON object to the file named by argv[1]: per
// test its status and, per source line, how many comparisons were evaluated
// and how many failed.  The tests' own console output goes to stdout.
#include <cstring>

#include "shim/refapi.h"

static std::string jsonEscape(const std::string& s) {
  std::string o;
  for (char c : s) {
    if (c == '"' || c == '\\') o += '\\';
    o += c;
  }
  return o;
}

int main(int argc, char** argv) {
  if (argc < 2) {
    std::fprintf(stderr, "usage: %s <out.json> [test name]\n", argv[0]);
    return 2;
  }
  FILE* out = std::fopen(argv[1], "w");
  if (!out) return 2;
  const char* only = argc > 2 ? argv[2] : nullptr;
  std::fprintf(out, "{\"tests\": [");
  bool first = true;
  for (const rt::Case& c : rt::registry()) {
    if (only && std::strcmp(only, c.name) != 0) continue;
    rt::state().test = c.name;
    std::string status = "ran", why;
    long long calls0 = rt::oracleCalls();
    try {
      c.fn();
    } catch (const rt::NotRestated& e) {
      status = "not_restated";
      why = e.what();
    }
    long long calls = rt::oracleCalls() - calls0;
    long long ev = 0, fail = 0;
    std::string lines;
    for (const auto& kv : rt::state().lines) {
      if (kv.first.first != c.name) continue;
      const rt::LineStat& s = kv.second;
      ev += s.evaluated;
      fail += s.failed;
      char buf[256];
      std::snprintf(buf, sizeof buf, "%s{\"line\": %d, \"kind\": \"%s\", \"evaluated\": %lld, \"failed\": %lld, "
                    "\"first_fail\": [%.9g, %.9g]}", lines.empty() ? "" : ", ", kv.first.second, s.kind.c_str(),
                    s.evaluated, s.failed, s.a, s.b);
      lines += buf;
    }
    std::fprintf(out, "%s\n {\"suite\": \"%s\", \"test\": \"%s\", \"status\": \"%s\", \"why\": \"%s\", "
                 "\"oracle_calls\": %lld, \"evaluated\": %lld, \"failed\": %lld, \"lines\": [%s]}", first ? "" : ",",
                 c.suite, c.name, status.c_str(), jsonEscape(why).c_str(), calls, ev, fail, lines.c_str());
    first = false;
  }
  std::fprintf(out, "\n]}\n");
  std::fclose(out);
  return 0;
}
