// CLI driver (the reference's include/prism.hpp:5 / src/prism.cu:9-192):
// compress, decompress and progressive-decompress flows with file I/O and the
// --report time,cr printouts.  Returns a process exit status.
#pragma once
#include "parameters.hpp"

int initialize(prism_context* config);
