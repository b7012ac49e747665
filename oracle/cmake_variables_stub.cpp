// ORACLE / TEST INFRASTRUCTURE ONLY.
// Definitions for the functions that the reference's CMake build generates from
// cieutils/src/cmake_variables.cpp.in (declared in cieutils/inc/cmake_variables.hpp:13-33).
// The reference solver sources link against them; the values do not affect any
// arithmetic.
#include <filesystem>
#include <string>

namespace cie {
std::filesystem::path getInstallPath() { return "."; }
std::filesystem::path getBinaryPath() { return "."; }
std::filesystem::path getSourcePath() { return "."; }
std::filesystem::path getDataPath() { return "."; }
std::filesystem::path getOutputPath() { return "."; }
bool isMPIEnabled() { return false; }
bool isSYCLEnabled() { return false; }
std::string getCompiler() { return "GNU"; }
std::string getCompilerVersion() { return __VERSION__; }
std::string getCompileFlags() { return ""; }
std::string getCompilePlatform() { return "Linux"; }
} // namespace cie
