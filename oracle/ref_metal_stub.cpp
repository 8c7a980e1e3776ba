// Stand-in for the reference's two Metal entry points (metal/taylor_green_backend.hpp:14-15),
// which need macOS and an Apple GPU.  Linked only into oracle/_ref/liborchard_ref.so, the
// test-only build of the reference's CPU path.
#include "metal/taylor_green_backend.hpp"

#include <stdexcept>

namespace solver::metal {

bool is_backend_available() {
  return false;
}

TaylorGreenMetalRun run_taylor_green(const TaylorGreenConfig&) {
  throw std::runtime_error("Metal backend is unavailable on this platform");
}

}  // namespace solver::metal
