// Internal handle types behind the C ABI.
#pragma once
#include <exception>
#include <new>
#include <string>

#include "gdtp.h"
#include "setup/setup.h"

struct gdtp_hierarchy {
  gdtp::Mesh mesh;
  int width = 0, height = 0;
  gdtp::Hierarchy h;
  gdtp::BoundaryElements be;
};

namespace gdtp {
extern thread_local std::string g_last_error;
int fail(int code, const std::string& msg);
int emit_csr(const Csr& m, const std::string& part, void* out, int64_t* count);

// Runs the body of a C entry point; a C++ exception (host allocation failure,
// a container length error) becomes an error code and gdtp_last_error() text
// instead of unwinding into C callers, which would end the process.
template <class Body>
int guarded(const char* entry, Body&& body) noexcept {
  try {
    return body();
  } catch (const std::bad_alloc&) {
    return fail(GDTP_ERR_SETUP, std::string(entry) + ": out of host memory");
  } catch (const std::exception& e) {
    return fail(GDTP_ERR_INVALID, std::string(entry) + ": " + e.what());
  } catch (...) {
    return fail(GDTP_ERR_INVALID, std::string(entry) + ": unexpected exception");
  }
}
}  // namespace gdtp
