// Host-side helpers shared by the C ABI translation units.
#pragma once

#include "gamera_op.h"

namespace gop {
// validates a descriptor (0 or a GOP_E* code with the message set)
int check_desc(const gop_desc* d);
// sets the thread's last-error message and returns code
int set_error(int code, const char* fmt, ...);
}  // namespace gop
