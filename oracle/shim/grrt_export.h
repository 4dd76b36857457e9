/* Stand-in for the export header that the reference's CMake build generates
 * (GenerateExportHeader). Only used to compile the reference sources under
 * oracle/_ref. */
#pragma once
#define GRRT_EXPORT __attribute__((visibility("default")))
#define GRRT_NO_EXPORT __attribute__((visibility("hidden")))
