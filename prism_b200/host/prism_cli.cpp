// prism command-line tool (the reference's examples/prism.cpp).
#include "parameters.hpp"
#include "prism.hpp"

int main(int argc, char* argv[]) {
  prism_context config;
  if (parse_argv(&config, argc, argv)) return 1;
  if (!config.isComp && !config.isDecomp) return 0;
  return initialize(&config);
}
