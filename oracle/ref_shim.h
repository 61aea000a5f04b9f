/*
 * ref_shim.h -- TEST INFRASTRUCTURE ONLY.  Force-included (g++ -include) into
 * every translation unit of the reference when oracle/build_ref.sh compiles it.
 *
 * The reference bakes its configuration directory (SOURCE_DIR, one per module)
 * and its output directory (DATA_DIR) into the binary as string macros
 * (CMakeLists.txt:46-49, Core/CMakeLists.txt:24-27).  Here both become calls
 * that read GFT_REF_WORKDIR at run time, so one binary can run any generated
 * configuration:
 *     SOURCE_DIR -> $GFT_REF_WORKDIR/<Module>     (configs in <Module>/Config/)
 *     DATA_DIR   -> $GFT_REF_WORKDIR/Data
 * The reference sources themselves are compiled unmodified.
 *
 * With -DGFT_REF_FP64 the shim also turns every `float` into `double` (and
 * powf into std::pow) after all standard headers have been included: the
 * FP64-storage variant of the reference.
 */
#ifndef GFT_REF_SHIM_H
#define GFT_REF_SHIM_H

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <random>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

static inline std::string gft_ref_workdir()
{
    const char* w = std::getenv("GFT_REF_WORKDIR");
    return w ? std::string(w) : std::string(".");
}

#ifdef GFT_REF_MODULE
#define GFT_REF_STR2(x) #x
#define GFT_REF_STR(x) GFT_REF_STR2(x)
#define SOURCE_DIR (gft_ref_workdir() + "/" GFT_REF_STR(GFT_REF_MODULE))
#endif
#define DATA_DIR (gft_ref_workdir() + "/Data")

#ifdef GFT_REF_FP64
#define float double
#define powf std::pow
#endif

#endif
