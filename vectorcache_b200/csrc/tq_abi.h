// Error plumbing shared by the C ABI translation units: nothing throws across
// the boundary; each entry point runs its body through guarded(), which maps
// exceptions to TQ_ERR_* codes and keeps the message per thread.
#pragma once

#include <new>
#include <stdexcept>
#include <string>

#include "../../include/vectorcache_b200.h"

namespace vcb {

// Defined once in tq_index.cu.
extern thread_local std::string g_last_error;

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] inline void fail(int code, const std::string& msg) { throw Error(code, msg); }

inline void require(bool ok, int code, const char* msg) {
  if (!ok) fail(code, msg);
}

template <typename F>
int guarded(F&& f) {
  try {
    f();
    g_last_error.clear();
    return TQ_OK;
  } catch (const Error& e) {
    g_last_error = e.what();
    return e.code;
  } catch (const std::bad_alloc&) {
    g_last_error = "host allocation failed";
    return TQ_ERR_OUT_OF_MEMORY;
  } catch (const std::exception& e) {
    g_last_error = e.what();
    return TQ_ERR_INVALID_ARGUMENT;
  } catch (...) {
    g_last_error = "unknown error";
    return TQ_ERR_CUDA;
  }
}

}  // namespace vcb
