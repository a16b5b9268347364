/* Stand-in for <openjpeg.h>: the integer types the reference's
 * snapshotmanager.h names in member declarations.  The frame harness
 * compiles no JPEG 2000 code. */
#pragma once
#include <cstddef>
#include <cstdint>
typedef size_t OPJ_SIZE_T;
typedef int64_t OPJ_OFF_T;
typedef int OPJ_BOOL;
