// imag3d-mpicuda: imaginary-time propagation (ground state), drop-in for the
// reference program of the same name (src/imag3d-mpicuda/imag3d-mpicuda.cu).
#include "cli.h"

int main(int argc, char **argv) { return gpecli::run_program(0, argc, argv); }
