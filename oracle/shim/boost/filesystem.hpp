// Test-infrastructure shim: the Boost.Filesystem calls the reference's IO layer
// makes, forwarded to std::filesystem (C++17).
#pragma once
#include <filesystem>

namespace boost {
namespace filesystem {
using path = std::filesystem::path;
inline bool exists(const path& p) { return std::filesystem::exists(p); }
inline bool is_regular_file(const path& p) { return std::filesystem::is_regular_file(p); }
inline bool is_directory(const path& p) { return std::filesystem::is_directory(p); }
inline bool create_directories(const path& p) { return std::filesystem::create_directories(p); }
} // namespace filesystem
} // namespace boost
