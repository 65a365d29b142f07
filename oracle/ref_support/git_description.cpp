// Test infrastructure (oracle build only): the build-time commit string the reference's CMake
// generates (src/app/git_description.hpp); this out-of-tree build has no commit to describe.
#include "app/git_description.hpp"

namespace spodvr {
std::string_view git_description() { return "oracle-build"; }
}  // namespace spodvr
