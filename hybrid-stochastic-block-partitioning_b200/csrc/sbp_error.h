// Last-error text of the C ABI (sbp_last_error in include/sbp_b200.h), shared by the
// library's translation units.  The text lives in a fixed per-thread buffer, so recording a
// failure allocates nothing (the allocation-free entry point reports through it too).
#pragma once

namespace sbpb {

// Record `msg` (truncated to the buffer) as the calling thread's last failure.
void set_last_error(const char* msg);
// The calling thread's last failure ("" before the first one).
const char* last_error();

}  // namespace sbpb
