// mph_io.h — host-side writers shared by the C ABI and the command-line driver.
#pragma once

namespace mph {

// writeVtkFile (main.cpp:698-834) from host arrays in the caller's order.
int write_vtk_host(const char* path, int n, const int* type, const double* xyz, const double* vel,
                   const double* force, const int* ncount, const double* dens_a, const double* strain_p,
                   const double* virial_p);

}  // namespace mph
