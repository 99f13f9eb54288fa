// Entry point of the PRISM flows (include/prism.hpp:5 of the reference):
// initialize runs what the prism_context asks for -- compress, decompress,
// or progressive decompress with its list of target errors -- reading and
// writing the files it names and printing the --report lines.
#pragma once
#include "parameters.hpp"

// Failures print the reason and end the process, as in the reference.
void initialize(prism_context* config);
// The same, returning 0 on success and nonzero after printing the reason.
int prism_initialize(prism_context* config);
