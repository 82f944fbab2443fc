// StaConfig.hh — stand-in for the header the reference's CMake build writes
// from util/StaConfig.hh.cmake (configure_file, CMakeLists.txt:425-426).
// The reference helpers compiled by oracle/Makefile (target `ref`) read
// none of these values; they exist so that include/sta/Delay.hh compiles.
// SSTA 0 selects the scalar (non-statistical) delay type, as the default
// build does.
#pragma once
#define STA_VERSION "oracle-ref"
#define STA_GIT_SHA1 "none"
#define SSTA 0
#define TCL_READLINE 0
