// Host checks of the server's HBM admission policy (compiled and run by
// tests/test_serving_policy.py).
#include <cstdio>
#include <vector>

#include "server_policy.h"

#define CHECK(c)                                              \
  do {                                                        \
    if (!(c)) {                                               \
      std::printf("FAIL line %d: %s\n", __LINE__, #c);        \
      return 1;                                               \
    }                                                         \
  } while (0)

int main() {
  using gdtp::AdmissionPolicy;
  AdmissionPolicy p(100);
  std::vector<int> v;
  CHECK(p.plan(60, v) && v.empty());
  p.add(1, 60, 1);
  CHECK(p.used() == 60 && p.peak() == 60);
  CHECK(p.plan(40, v) && v.empty());
  p.add(2, 40, 2);
  CHECK(p.used() == 100);
  // needs room: least recently used idle model goes first
  CHECK(p.plan(30, v) && v.size() == 1 && v[0] == 1);
  p.set_busy(1, true, 3);  // 1 now busy and most recent
  CHECK(p.plan(30, v) && v.size() == 1 && v[0] == 2);
  p.set_busy(2, true, 4);
  CHECK(!p.plan(30, v) && v.empty());  // everything busy
  p.set_busy(1, false, 5);
  p.set_busy(2, false, 6);
  CHECK(p.plan(100, v) && v.size() == 2 && v[0] == 1 && v[1] == 2);
  CHECK(!p.plan(101, v));               // larger than the budget
  CHECK(p.plan(40, v, 1) && v.size() == 1 && v[0] == 2);  // excluded model is never a victim
  CHECK(!p.plan(50, v, 1));
  p.evict(2);
  CHECK(p.used() == 60 && p.evictions() == 1 && !p.resident(2) && p.resident(1));
  p.add(1, 80, 7);                      // re-measured size replaces the estimate
  CHECK(p.used() == 80 && p.peak() == 100);
  std::printf("ok\n");
  return 0;
}
