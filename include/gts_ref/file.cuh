// file.cuh -- stands in for the reference header of this name (Source Code/GTS/include/file.cuh):
// its entry points come from gts_ref_compat.h over libgts_b200.  Like the
// reference's headers it brings the std namespace in (the reference's
// src/main.cu calls stod unqualified).
#pragma once
#include <chrono>
#include <string>
#include "../gts_ref_compat.h"
using namespace std;
