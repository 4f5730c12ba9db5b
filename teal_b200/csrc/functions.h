// Registry of device functions compiled at run time (functions.cu).
#pragma once

#include <string>

namespace tg {

enum { FUNCTION_BOUNDARY = 1, FUNCTION_SOURCE = 2 };

// Compile and register `source` under `name`. Returns 0, 1 (invalid argument or a compile error:
// the compiler log goes to `log`) or 2 (NVRTC unavailable); `error` says which.
int function_register(const char *name, int kind, const char *source, char *log, long log_size,
                      std::string &error);

// The kernel of a registered function of `kind`, loaded on first use (needs a device). Returns 0,
// 1 (not registered / other kind) or 2 (load failure).
int function_kernel(const char *name, int kind, const void **kernel, std::string &error);

}  // namespace tg
