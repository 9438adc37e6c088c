// Configured version header for compiling the reference's headers into the
// CPU checker (the reference generates this file from config.hpp.in at
// configure time; MCNLA 0.7.2 per its CMakeLists.txt).
#ifndef MCNLA_CONFIG_HPP_
#define MCNLA_CONFIG_HPP_

#define MCNLA_MAJOR_VERSION 0
#define MCNLA_MINOR_VERSION 7
#define MCNLA_PATCH_VERSION 2

#endif  // MCNLA_CONFIG_HPP_
