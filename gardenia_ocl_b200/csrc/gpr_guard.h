// Guard for the bodies of C entry points: a C++ exception from host code
// (out of host memory in a std::vector, a thread that cannot start) becomes a
// gpr_status with a message instead of crossing the C boundary, where it would
// end the caller's process.  Exceptions of any type are caught.
//
//   int gpr_x(...) {
//     GPR_ENTRY_BEGIN
//     ... body, returning a status on every path ...
//     GPR_ENTRY_END("gpr_x")
//   }
#ifndef GPR_GUARD_H_
#define GPR_GUARD_H_

#include <exception>
#include <new>

#include "gpr.h"

namespace gpr {
void set_error(const char *fmt, ...);
}

#define GPR_ENTRY_BEGIN try {
#define GPR_ENTRY_END(name)                                                   \
  }                                                                           \
  catch (const std::bad_alloc &) {                                            \
    gpr::set_error("%s: out of host memory", name);                           \
    return GPR_ENOMEM;                                                        \
  }                                                                           \
  catch (const std::exception &e_) {                                          \
    gpr::set_error("%s: %s", name, e_.what());                                \
    return GPR_EINVAL;                                                        \
  }                                                                           \
  catch (...) {                                                               \
    gpr::set_error("%s: unknown host exception", name);                       \
    return GPR_EINVAL;                                                        \
  }

#endif  // GPR_GUARD_H_
