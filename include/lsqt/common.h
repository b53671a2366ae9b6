// C++ drop-in surface of the LSQT hot path: the reference's classes and functions
// (src/common.h, src/model.h, src/hamiltonian.h, src/vector.h, src/sigma.h,
// src/lsqt.h) over the C ABI in gpuqt.h. Failures print a message and exit(1), as
// the reference does; the C ABI underneath returns status codes instead.
#pragma once

#include <stdexcept>
#include <string>

typedef double real;  // src/common.h:22-26 (the FP32 form is a runtime choice here)

namespace gqt_host {
// Raised by the model builder; the public constructors turn it into print + exit(1).
struct InputError : std::runtime_error {
  using std::runtime_error::runtime_error;
};
// Raised instead of exiting while a ThrowScope is active (the C-ABI driver entry
// points use one so that a failed run returns a status).
struct RunError : std::runtime_error {
  int code;
  RunError(const std::string& m, int c) : std::runtime_error(m), code(c) {}
};
struct ThrowScope {
  ThrowScope();
  ~ThrowScope();
  bool saved;
};
// Print + exit(1) (or throw RunError inside a ThrowScope).
[[noreturn]] void die(const std::string& message, int code = 4);
// die() with the library's last error message when status != 0.
void check(int status, const char* what);
// Records a message for gqt_last_error().
void set_error(const std::string& message);
}  // namespace gqt_host
