// Build shim for compiling the reference sources in the oracle harness:
// the reference uses boost::filesystem only for path joining and directory
// creation, which std::filesystem provides.
#pragma once
#include <filesystem>
namespace boost { namespace filesystem = std::filesystem; }
