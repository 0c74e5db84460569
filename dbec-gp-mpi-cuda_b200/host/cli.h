// cli.h -- the imag3d-mpicuda / real3d-mpicuda programs on top of the C ABI.
#pragma once

namespace gpecli {

// mode: 0 = imaginary time (imag3d-mpicuda), 1 = real time (real3d-mpicuda).
// Returns the process exit status.
int run_program(int mode, int argc, char **argv);

}  // namespace gpecli
