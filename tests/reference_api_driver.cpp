/*
 * reference_api_driver.cpp -- a caller written against the reference's C++ API
 * (include/lt_reference_api.hpp), linked against liblt_b200.so by
 * tests/test_reference_api.py.
 *
 * Input file (binary): int n; int type[n]; double x, y, b0, angle, cos, sin, eps, rcore,
 * rcut, dlsds [n each]; double frame[4] (xmin xmax ymin ymax); int nbgridcells.
 * Output file (binary, nbgridcells^2 doubles each): ax, ay, a, b, c, d, ampli1, ampli5,
 * shear4, mass2, pot1, dplx, dply, hess_a via *_CPU_GPU on device buffers.
 */
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "lt_reference_api.hpp"

static void rd(FILE *f, void *p, size_t n)
{
    if (fread(p, 1, n, f) != n) {
        fprintf(stderr, "short read\n");
        exit(2);
    }
}

int main(int argc, char **argv)
{
    if (argc != 3) return 2;
    FILE *f = fopen(argv[1], "rb");
    if (!f) return 2;
    int n;
    rd(f, &n, sizeof(int));
    std::vector<int> type(n + 1, -1);
    rd(f, type.data(), sizeof(int) * n);
    std::vector<double> a[10];
    for (auto &v : a) {
        v.resize(n);
        rd(f, v.data(), sizeof(double) * n);
    }
    double fr[4];
    rd(f, fr, sizeof(fr));
    int ng;
    rd(f, &ng, sizeof(int));
    fclose(f);

    Potential_SOA lens;
    memset(&lens, 0, sizeof(lens));
    std::vector<double> z(n, 0.35);
    lens.type = type.data();
    lens.position_x = a[0].data();
    lens.position_y = a[1].data();
    lens.b0 = a[2].data();
    lens.ellipticity_angle = a[3].data();
    lens.anglecos = a[4].data();
    lens.anglesin = a[5].data();
    lens.ellipticity_potential = a[6].data();
    lens.rcore = a[7].data();
    lens.rcut = a[8].data();
    lens.dlsds = a[9].data();
    lens.z = z.data();
    grid_param frame;
    memset(&frame, 0, sizeof(frame));
    frame.xmin = fr[0];
    frame.xmax = fr[1];
    frame.ymin = fr[2];
    frame.ymax = fr[3];
    cosmo_param cosmo;
    memset(&cosmo, 0, sizeof(cosmo));
    cosmo.model = 1;
    cosmo.omegaM = 0.3;
    cosmo.omegaX = 0.7;
    cosmo.wX = -1.;
    cosmo.H0 = 70.;
    cosmo.h = 70. / 50.;
    runmode_param rm;
    rm.amplif = 1;
    rm.shear = 4;
    rm.mass = 2;
    rm.potential = 1;

    const size_t np = (size_t)ng * ng;
    std::vector<std::vector<double>> out(14, std::vector<double>(np, 0.));
    gradient_grid_GPU(out[0].data(), out[1].data(), &frame, &lens, n, ng);
    gradient2_grid_GPU(out[2].data(), out[3].data(), out[4].data(), out[5].data(), &frame, &lens, n, ng);
    map_grid_ampli_GPU(select_map_ampli_function(&rm), out[6].data(), &cosmo, &frame, &lens, n, ng, 1, 1.5);
    rm.amplif = 5;
    map_grid_ampli_GPU(select_map_ampli_function(&rm), out[7].data(), &cosmo, &frame, &lens, n, ng, 5, 1.5);
    map_grid_shear_GPU(select_map_shear_function(&rm), out[8].data(), &cosmo, &frame, &lens, n, ng, 4, 1.5);
    map_grid_mass_GPU(select_map_mass_function(&rm), out[9].data(), &cosmo, &frame, &lens, n, ng, 2, 0.35, 1.5);
    map_grid_potential_GPU(select_map_potential_function(&rm), out[10].data(), &cosmo, &frame, &lens, n, ng, 1, 1.5);
    map_grid_dpl_GPU(nullptr, out[11].data(), out[12].data(), &cosmo, &frame, &lens, n, ng, 1, 1.5);

    /* the device-pointer launcher with a device-resident Potential_SOA and frame, as the
     * reference's map builders call it (src/grid_map_ampli_GPU.cu:119-165) */
    Potential_SOA dl = lens;
    int *dtype;
    cudaMalloc(&dtype, sizeof(int) * n);
    cudaMemcpy(dtype, type.data(), sizeof(int) * n, cudaMemcpyHostToDevice);
    dl.type = dtype;
    double *dfields[10];
    double **slots[10] = {&dl.position_x, &dl.position_y, &dl.b0, &dl.ellipticity_angle, &dl.anglecos,
                          &dl.anglesin, &dl.ellipticity_potential, &dl.rcore, &dl.rcut, &dl.dlsds};
    for (int k = 0; k < 10; k++) {
        cudaMalloc(&dfields[k], sizeof(double) * n);
        cudaMemcpy(dfields[k], a[k].data(), sizeof(double) * n, cudaMemcpyHostToDevice);
        *slots[k] = dfields[k];
    }
    Potential_SOA *dlens;
    grid_param *dframe;
    cudaMalloc(&dlens, sizeof(Potential_SOA));
    cudaMalloc(&dframe, sizeof(grid_param));
    cudaMemcpy(dlens, &dl, sizeof(dl), cudaMemcpyHostToDevice);
    cudaMemcpy(dframe, &frame, sizeof(frame), cudaMemcpyHostToDevice);
    double *planes;
    cudaMalloc(&planes, 4 * np * sizeof(double));
    module_potentialDerivatives_totalGradient2_SOA_CPU_GPU(planes, planes + np, planes + 2 * np, planes + 3 * np, dframe,
                                                           dlens, ng, n);
    cudaDeviceSynchronize();
    cudaMemcpy(out[13].data(), planes, np * sizeof(double), cudaMemcpyDeviceToHost);

    FILE *o = fopen(argv[2], "wb");
    for (auto &v : out) fwrite(v.data(), sizeof(double), np, o);
    fclose(o);
    return lt_reference_api_last_status();
}
