// Internal declarations shared by the host driver and the CUDA kernels of
// libsharp_b200.so.  Nothing here is part of the public ABI.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>

#include "sharp_lowlevel.h"
#include "sharp_b200.h"

namespace sht {

// ---------------------------------------------------------------------------
// Error handling.  The reference aborts the process on any precondition
// failure (c_utils/c_utils.c:35-39: message to stderr, exit(1)).  That stays
// the default; with sharp_b200_set_abort_on_error(0) (or the environment
// variable SHARP_B200_ABORT_ON_ERROR=0) the failing call returns early and
// the message is kept for sharp_b200_last_error().
// ---------------------------------------------------------------------------
struct Failure {
  std::string msg;
};

[[noreturn]] void fail(const char *file, int line, const std::string &msg);
void record_error(const std::string &msg);
bool abort_on_error();

#define SHT_REQUIRE(cond, msg) \
  do { if (!(cond)) ::sht::fail(__FILE__, __LINE__, (msg)); } while (0)

// Transform constants shared by host and device code.
constexpr int kMaxTrans = 100;          // SHARP_MAXTRANS, libsharp/sharp_internal.h:41
constexpr int kLBlock = 16;             // l-steps per Legendre block (even)
constexpr int kPad = 2 * kLBlock;       // zero padding after each m segment
constexpr int kSwitchExp = 200;         // recurrence values below 2^-200 are skipped

// Geometry helpers used by the device planner.
int get_mlim(int lmax, int spin, double sth, double cth);

}  // namespace sht
