// The C entry points' exception guard (csrc/capi_internal.h): an exception in
// an entry point's body becomes an error code and a message, never an unwind
// into the C caller.  Linked with the library, which defines fail() and the
// thread's last-error text.
#include <cstdio>
#include <new>
#include <stdexcept>
#include <string>

#include "capi_internal.h"

int main() {
  using gdtp::guarded;
  int bad = 0;
  auto expect = [&](int got, int code, const char* msg) {
    const std::string last = gdtp_last_error();
    if (got != code || last != msg) {
      std::printf("got %d '%s', want %d '%s'\n", got, last.c_str(), code, msg);
      bad++;
    }
  };
  expect(guarded("gdtp_a", []() -> int { throw std::bad_alloc(); }), GDTP_ERR_SETUP, "gdtp_a: out of host memory");
  expect(guarded("gdtp_b", []() -> int { throw std::length_error("vector too long"); }), GDTP_ERR_INVALID, "gdtp_b: vector too long");
  expect(guarded("gdtp_c", []() -> int { throw 7; }), GDTP_ERR_INVALID, "gdtp_c: unexpected exception");
  if (guarded("gdtp_d", []() -> int { return 3; }) != 3) bad++;
  std::printf(bad ? "failed\n" : "ok\n");
  return bad ? 1 : 0;
}
