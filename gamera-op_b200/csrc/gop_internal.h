// Host-side helpers shared by the C ABI translation units.
#pragma once

#include "gamera_op.h"

namespace gop {
// validates a descriptor (0 or a GOP_E* code with the message set)
int check_desc(const gop_desc* d);
// sets the thread's last-error message and returns code
int set_error(int code, const char* fmt, ...);
// the pole ring average of a descriptor: poles reached (bit 0 theta = 0,
// bit 1 theta = pi), ring rows per pole - 1, phi blocks per ring row
struct RingSetup {
  int poles = 0;
  int jmax = 0;
  int nchunk[16] = {0};
};
int ring_setup(const gop_desc* d, RingSetup& r);
}  // namespace gop
