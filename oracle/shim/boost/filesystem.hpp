// Stand-in for the un-vendored Boost.Filesystem submodule: the reference's
// plugin manager (src/core/plugin_manager.cpp) and path helpers
// (src/core/system/utf8_path.*) use only what std::filesystem provides under
// the same names (path, directory_iterator, filesystem_error).
#pragma once

#include <filesystem>

namespace boost
{
namespace filesystem = std::filesystem;
} // namespace boost
