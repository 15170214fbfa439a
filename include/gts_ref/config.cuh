// config.cuh -- stands in for the reference's config.cuh: the data type of
// numeric objects is float (Source Code/GTS/include/config.cuh:5 defines
// short as float, and the reference's programs declare their rows short).
#pragma once
#define short float
