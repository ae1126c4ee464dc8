// common.h -- shared host-side declarations of the backend.
#pragma once
#include <cstdarg>
#include <cstdint>
#include "bnc_abi.h"
#include "bnc_b200.h"

namespace bnc {
// Records the message returned by bnc_last_error() on this thread.
void set_error(const char* fmt, ...);
}  // namespace bnc
