/* A plain C99 consumer of the C ABI (include/cfdgpu.h, include/cfdgpu_host.h):
 * what an FFI binding or a C host program sees.  Builds a configuration and
 * an initial condition on the host, then asks for a solver; prints one line
 * per call.  Without a CUDA device the solver call must fail with
 * CFD_ERR_CUDA and a message, never fall back to the CPU. */
#include <stdio.h>
#include <stdlib.h>

#include "cfdgpu.h"
#include "cfdgpu_host.h"

int main(void) {
    cfd_config cfg;
    cfd_solver* solver = NULL;
    size_t elems = 0;
    double* grid;
    char msg[256];
    int rc;

    printf("version %s\n", cfd_version());
    rc = cfd_recipe_config(CFD_RECIPE_FOUR_QUADRANT, 32, 24, &cfg);
    printf("recipe_config %d nx %d ny %d\n", rc, cfg.nx, cfg.ny);
    if (rc) return 1;
    rc = cfd_ic_grid_elems(&cfg, &elems);
    printf("grid_elems %d %zu\n", rc, elems);
    grid = (double*)malloc(elems * sizeof(double));
    if (!grid) return 1;
    rc = cfd_recipe_ic(&cfg, CFD_RECIPE_FOUR_QUADRANT, 1, 0, grid);
    printf("recipe_ic %d first_rho %.17g\n", rc, grid[(2 * (cfg.nx + 4) + 2) * 4]);
    rc = cfd_create(&cfg, &solver);
    cfd_last_error(msg, sizeof msg);
    printf("create %d %s\n", rc, msg);
    if (rc == CFD_OK) {
        rc = cfd_upload(solver, grid, CFD_LAYOUT_GHOSTED_AOS, 0, 0.0);
        printf("upload %d\n", rc);
        cfd_destroy(solver);
    }
    free(grid);
    return 0;
}
