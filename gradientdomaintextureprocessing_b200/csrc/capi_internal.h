// Internal handle types behind the C ABI.
#pragma once
#include <string>

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
}  // namespace gdtp
