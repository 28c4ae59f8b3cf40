/* A plain C caller of the library's host-only entry points, as a program in
 * the reference's own languages would call them: read a *.data and a *.grid,
 * derive the set-up constants, write a VTK from host arrays, and let
 * mph_create reject a bad argument before it touches any device.  Built and
 * run by tests/test_c_abi.py; prints one line per result. */
#include <stdio.h>
#include <stdlib.h>

#include "mph_b200.h"

int main(int argc, char** argv) {
    if (argc != 5) {
        fprintf(stderr, "usage: c_abi_probe case.data case.grid out.vtk dim\n");
        return 2;
    }
    const int dim = atoi(argv[4]);
    mph_params p;
    int invalid = 0;
    if (mph_read_data_file(argv[1], &p, &invalid) != MPH_OK) return 1;
    mph_grid_header h;
    if (mph_read_grid_header(argv[2], &h) != MPH_OK) return 1;
    const int n = h.particle_count;
    int* type = (int*)calloc((size_t)n, sizeof(int));
    int* zeros_i = (int*)calloc((size_t)n, sizeof(int));
    double* xyz = (double*)calloc(3 * (size_t)n, sizeof(double));
    double* vel = (double*)calloc(3 * (size_t)n, sizeof(double));
    double* zeros = (double*)calloc(3 * (size_t)n, sizeof(double));
    if (!type || !zeros_i || !xyz || !vel || !zeros) return 1;
    if (mph_read_grid_file(argv[2], &h, n, type, xyz, vel) != MPH_OK) return 1;
    mph_constants c;
    if (mph_compute_constants(&p, &h, dim, &c) != MPH_OK) return 1;
    printf("particles %d invalid_lines %d dt %.17g\n", n, invalid, p.dt);
    printf("cells %d %d %d total %d\n", c.cell_count[0], c.cell_count[1], c.cell_count[2], c.total_cell_count);
    printf("max_radius %.17g\n", c.max_radius);
    /* writeVtkFile from host arrays: velocity doubles as the force column */
    printf("write_vtk %d\n", mph_write_vtk_arrays(argv[3], n, type, xyz, vel, vel, zeros_i, zeros, zeros, zeros));
    mph_ctx* ctx = NULL;
    const int st = mph_create(&p, &h, 4, MPH_MODE_FP64, type, xyz, vel, &ctx);
    char msg[256] = {0};
    mph_last_error(NULL, msg, (int)sizeof(msg));
    printf("create_dim4 %d ctx_null %d\n", st, ctx == NULL);
    printf("error_message %s\n", msg);
    free(type);
    free(zeros_i);
    free(xyz);
    free(vel);
    free(zeros);
    return 0;
}
