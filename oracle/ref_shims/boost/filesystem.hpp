// Test-infrastructure shim (oracle build only): boost::filesystem -> std::filesystem.
#pragma once
#include <filesystem>
namespace boost {
namespace filesystem = std::filesystem;
}
