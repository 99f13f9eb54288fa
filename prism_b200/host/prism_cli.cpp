// prism command-line tool: the flow of the reference's examples/prism.cpp
// (parse the flags, run the configured flows) with an exit status.
#include "parameters.hpp"
#include "prism.hpp"

int main(int argc, char* argv[]) {
  prism_context config;
  if (prism_parse_argv(&config, argc, argv)) return 1;
  if (!config.isComp && !config.isDecomp) return 0;
  return prism_initialize(&config);
}
