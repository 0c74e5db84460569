// real3d-mpicuda: real-time propagation (dynamics), drop-in for the reference
// program of the same name (src/real3d-mpicuda/real3d-mpicuda.cu).
#include "cli.h"

int main(int argc, char **argv) { return gpecli::run_program(1, argc, argv); }
