// Message of the last failed C-ABI call (ostc_last_error), per host thread.
#include <string>

namespace ostc {
namespace {
thread_local std::string g_error;
}

int abi_error(int code, const std::string &msg) {
  g_error = msg;
  return code;
}

const char *abi_last_error() { return g_error.c_str(); }
}  // namespace ostc
