// Common header of the <lslab/...> include shims.  Besides the C++ front it
// brings the standard headers that the reference's own headers provide to
// their callers through thrust and the CUDA headers (streams, chrono and
// the C library), since callers such as benchmark/benchmark.cu use them
// without including them.
#pragma once
#include <chrono>
#include <cstdlib>
#include <iostream>

#include "../lslab_compat.h"
